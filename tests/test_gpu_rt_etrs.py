"""The real-time loop under a self-consistent potential with both of the
reference's propagators (dt_evolve_KB, RT/dt_evolve.f90:28-63): 'middlepoint'
and 'etrs' (two half steps around the potential extrapolated from its history,
:218-348), on the GPU through the C ABI against the CPU oracle's loop
(oracle/rt_oracle.py).

Tolerances: orbitals 1e-11 relative (complex(8), a few steps of FP64 FFTs and
Taylor steps), J(t) 1e-10 relative to max |J|, Vloc 1e-11; complex(4) orbitals
2e-6 per step, J 1e-5 (the FP32+FP64-reduce target)."""
import numpy as np
import pytest

from _helpers import rel
from oracle import rt_oracle as RO
from salmon_b200 import drive, system as S

pytestmark = pytest.mark.gpu


def _case():
    sysm, kAc, vpsl, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (2, 1, 1), 8)
    kAc0 = np.ascontiguousarray(sysm.kAc0)
    # a strong, short Acos2 pulse so that k+A, the density and Vloc all move
    Ac = drive.init_Ac(8, 0.08, "Acos2", epdir=(0.0, 0.0, 1.0), rlaser_int_wcm2=1e15, omega=0.3, pulse_tw=1.0)
    return sysm, kAc0, vpsl, zu, Ac


@pytest.mark.parametrize("propagator", ["middlepoint", "etrs"])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_rt_loop_matches_oracle(cuda_lib, propagator, precision):
    from salmon_b200.rt import GpuSystem
    sysm, kAc0, vpsl, zu, Ac = _case()
    nt, dt = 4, 0.08
    z_in = zu if precision == "c128" else zu.astype(np.complex64).astype(np.complex128)
    z_ref, j_ref, v_ref = RO.rt_propagate(sysm, kAc0, vpsl, Ac, dt, nt, z_in, propagator)
    with GpuSystem(sysm, precision) as g:
        g.set_state(zu)
        g.update_projector(kAc0)
        javt, _ = drive.rt_propagate(g, sysm, kAc0, vpsl, Ac, dt, nt, scf=True, propagator=propagator)
        z = g.get_state()
        v = g.get_vloc()
    assert np.abs(j_ref).max() > 1e-6
    if precision == "c128":
        assert rel(z, z_ref) < 1e-11
        assert rel(javt, j_ref) < 1e-10
        assert rel(v, v_ref) < 1e-11
    else:
        assert rel(z, z_ref) < 2e-6 * nt
        assert rel(javt, j_ref) < 1e-5


def test_extrapolation_of_a_fixed_potential_is_the_potential(cuda_lib):
    """With the history reset to Vloc, 3 V - 3 V + V = V (to rounding): etrs under
    a fixed potential is two half Taylor steps."""
    from salmon_b200.rt import GpuSystem
    sysm, kAc0, vpsl, zu, Ac = _case()
    with GpuSystem(sysm, "c128") as g:
        g.set_vloc(vpsl)
        g.vloc_history_reset()
        for _ in range(2):
            g.vloc_extrapolate()
            assert np.abs(g.get_vloc() - vpsl).max() <= 1e-14 * np.abs(vpsl).max()
