"""Ground-state and real-time drivers over the C ABI.

These follow the control flow of SALMON's ARTED drivers with the potential
held fixed (no Hartree / exchange-correlation update between steps):

  init_Ac          RT/init_Ac.f90:17-100      A_ext(t) of 'impulse' and 'Acos<n>' pulses
  ground_state     control/ground_state.f90:100-150  Gram-Schmidt, subspace diag,
                                              Gram-Schmidt, CG, Gram-Schmidt per iteration
  rt_propagate     control/control_sc.f90:150-230 with dt_evolve_KB 'middlepoint'
                   (RT/dt_evolve.f90:45-49): k+A at the midpoint for the Taylor step,
                   k+A(t+dt) for the current
"""
from __future__ import annotations

import numpy as np

F0_PER_SQRT_WCM2 = 5.338e-9  # electric field in a.u. per sqrt(W/cm^2) (init_Ac.f90:34)


def init_Ac(Nt: int, dt: float, shape: str = "impulse", epdir=(1.0, 0.0, 0.0), e_impulse: float = 1e-3,
            rlaser_int_wcm2: float = 1e12, omega: float = 0.05696144984638035, pulse_tw: float = 110.0,
            phi_cep: float = 0.0, t_delay: float = 0.0):
    """Ac_ext(iter) for iter = -1..Nt+1 as an array of shape (Nt+3, 3); row
    iter+1 holds time iter*dt (RT/init_Ac.f90:44-84)."""
    ep = np.asarray(epdir, dtype=np.float64)
    Ac = np.zeros((Nt + 3, 3))
    if shape == "impulse":
        Ac[:, :] = ep * e_impulse
        return Ac
    if not shape.startswith("Acos"):
        raise ValueError(f"unsupported pulse shape {shape!r}")
    npower = int(shape[4:])
    f0 = F0_PER_SQRT_WCM2 * np.sqrt(rlaser_int_wcm2)
    for it in range(-1, Nt + 2):
        tt = it * dt - 0.5 * pulse_tw - t_delay
        if abs(tt) < 0.5 * pulse_tw:
            Ac[it + 1] = -f0 / omega * np.cos(np.pi * tt / pulse_tw) ** npower * np.imag(
                ep * np.exp(1j * (omega * tt + phi_cep * 2 * np.pi)))
    return Ac


def ground_state(g, n_iter: int = 4, ncg: int = 4):
    """Iterations of the ground-state sequence at fixed potential on the device
    ground-state orbitals; returns (esp (nkl,NB), esp_var (nkl,NB), history)
    with history[i] = (sum of esp, max of esp_var) after iteration i."""
    esp = esp_var = None
    history = []
    for _ in range(n_iter):
        g.gram_schmidt()
        esp = g.subspace_diag()
        g.gram_schmidt()
        esp_var, _ = g.cg(ncg)
        g.gram_schmidt()
        history.append((float(esp.sum()), float(esp_var.max())))
    esp = g.subspace_diag()
    return esp, esp_var, history


def band_energy(g, sysm, kAc, vloc):
    """Ekin + Enl + sum_i Vloc_i rho_i Hxyz of the resident orbitals (FP64)."""
    ek, en = g.energy_terms(kAc)
    rho = g.psi_rho_RT()
    return ek + en + float(np.dot(vloc, rho)) * sysm.Hxyz


def rt_propagate(g, sysm, kAc0, vloc, Ac, dt: float, Nt: int, energy_every: int = 0):
    """Nt middle-point Taylor steps of the resident orbitals; returns
    (javt (Nt+1,3) with javt[0] the current before the first step,
     energies {step: band energy} every `energy_every` steps)."""
    kAc0 = np.ascontiguousarray(kAc0, dtype=np.float64)
    g.set_vloc(vloc)
    javt = np.zeros((Nt + 1, 3))
    javt[0] = g.current_RT(kAc0 + Ac[1][:, None])
    energies = {}
    if energy_every:
        energies[0] = band_energy(g, sysm, kAc0 + Ac[1][:, None], vloc)
    for it in range(Nt):
        kmid = kAc0 + 0.5 * (Ac[it + 1] + Ac[it + 2])[:, None]   # kAc0 + (Ac(it)+Ac(it+1))/2
        g.update_projector(kmid)
        g.hamiltonian(dt)
        knew = kAc0 + Ac[it + 2][:, None]
        javt[it + 1] = g.current_RT(knew)
        if energy_every and (it + 1) % energy_every == 0:
            energies[it + 1] = band_energy(g, sysm, knew, vloc)
    return javt, energies


def j_error(j_ref, j_test):
    """max_t |J_test(t) - J_ref(t)| / max_t |J_ref(t)|, per component maximum."""
    j_ref = np.asarray(j_ref)
    j_test = np.asarray(j_test)
    return float(np.abs(j_test - j_ref).max() / np.abs(j_ref).max())


def j_error_dynamic(j_ref, j_test):
    """The same error relative to the time-dependent part of J (J(t) - J(0))."""
    d_ref = np.asarray(j_ref) - np.asarray(j_ref)[0]
    d_test = np.asarray(j_test) - np.asarray(j_test)[0]
    return float(np.abs(d_test - d_ref).max() / max(np.abs(d_ref).max(), 1e-300))
