"""CPU oracle of SALMON's real-time loop with the self-consistent potential:
the middle-point and etrs propagators.  TEST INFRASTRUCTURE ONLY.

  middlepoint   RT/dt_evolve.f90:45-49, :104-207 (dt_evolve_omp_KB): one Taylor
                step of dt at kAc0 + (A(t) + A(t+dt))/2, then rho, Vloc = Vh + Vpsl
                + Vexc
  etrs          RT/dt_evolve.f90:53-63, :218-348 (dt_evolve_etrs_omp_KB, LDA
                functionals): a Taylor step of dt/2 at kAc0 + A(t); Vloc_new =
                3 Vloc - 3 Vloc_old(:,1) + Vloc_old(:,2), Vloc_old(:,2) =
                Vloc_old(:,1), Vloc_old(:,1) = Vloc, Vloc = Vloc_new; a Taylor step
                of dt/2 at kAc0 + A(t+dt); then rho, Vloc = Vh + Vpsl + Vexc.  The
                history starts as Vloc_old(:,1) = Vloc_old(:,2) = Vloc
                (control/control_sc.f90:82).
  current       after every step at kAc0 + A(t+dt) (control_sc.f90:203-209).

The Taylor step, projectors, density and current are the C restatement
(oracle.hamiltonian etc.); Hartree and PZ are scf_oracle."""
from __future__ import annotations

import numpy as np

from . import oracle as O
from . import scf_oracle as X


def rt_propagate(sysm, kAc0, vpsl, Ac, dt, Nt, zu, propagator="middlepoint"):
    """Returns (zu after Nt steps, javt (Nt+1, 3), Vloc after the last step)."""
    shape = (sysm.NLx, sysm.NLy, sysm.NLz)
    kAc0 = np.ascontiguousarray(kAc0, dtype=np.float64)
    z = np.array(zu, dtype=np.complex128, copy=True)
    v, _ = X.vloc(O.psi_rho(sysm, z), vpsl, shape, sysm.aL, sysm.Hxyz)
    h1 = v.copy()
    h2 = v.copy()
    javt = np.zeros((Nt + 1, 3))
    javt[0] = O.current(sysm, np.ascontiguousarray(kAc0 + Ac[1][:, None]), z)
    for it in range(Nt):
        kt = np.ascontiguousarray(kAc0 + Ac[it + 1][:, None])
        knew = np.ascontiguousarray(kAc0 + Ac[it + 2][:, None])
        if propagator == "middlepoint":
            kmid = np.ascontiguousarray(kAc0 + 0.5 * (Ac[it + 1] + Ac[it + 2])[:, None])
            _, zp = O.update_projector(sysm, kmid)
            z = O.hamiltonian(sysm, kmid, v, zp, dt, z)
        elif propagator == "etrs":
            _, zp = O.update_projector(sysm, kt)
            z = O.hamiltonian(sysm, kt, v, zp, 0.5 * dt, z)
            vnew = 3.0 * v - 3.0 * h1 + h2
            h2 = h1
            h1 = v
            v = vnew
            _, zp = O.update_projector(sysm, knew)
            z = O.hamiltonian(sysm, knew, v, zp, 0.5 * dt, z)
        else:
            raise ValueError(propagator)
        v, _ = X.vloc(O.psi_rho(sysm, z), vpsl, shape, sysm.aL, sysm.Hxyz)
        javt[it + 1] = O.current(sysm, knew, z)
    return z, javt, v
