"""The shared-memory resident Taylor step (one CTA holds an orbital for the
whole step: 16x16, 16x32 and 20x20 planes) and the current computed with the
step (flag_current), against the CPU oracle.

Tolerances (max |gpu - oracle| / max |oracle|): complex(8) 1e-12 per step,
complex(4) 2e-6 per step; the current 1e-12 against the oracle on the same
orbitals; the resident and the stencil-pass forms of the step agree to 1e-13
(complex(8))."""
import os

import numpy as np
import pytest

from _helpers import GOLDEN, rel
from oracle import oracle as O
from salmon_b200 import pseudo as P, system as S

pytestmark = pytest.mark.gpu
TOL = {"c128": 1e-12, "c64": 2e-6}


def _si_pp16():
    tabs = P.prepare(P.from_npz(os.path.join(GOLDEN, "si_rps_ky.npz"), lloc=2))
    sysm, kAc0, vpsl, zu = S.si_pp_system(tabs, grid=(16, 16, 16), nkgrid=(2, 1, 1), NB=16, Nocc=16)
    return sysm, np.ascontiguousarray(kAc0 + np.array([1e-2, 0.0, 0.0])[:, None]), vpsl, zu


CASES = {
    "microbench_16": lambda: S.microbench_system(16, nk_limit=2, Nb=8),
    "microbench_20": lambda: S.microbench_system(20, nk_limit=1, Nb=8),
    "si16_16x16x32": lambda: S.si_supercell_system((1, 1, 2), (16, 16, 32), (1, 1, 1), 12, A=(0.0, 0.0, 1e-2)),
    "si8_pseudopotential_16": _si_pp16,
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, cuda_lib):
    return (request.param,) + tuple(CASES[request.param]())


def _gpu(sysm, kAc, vloc, zu, precision, kernel):
    from salmon_b200.rt import GpuSystem
    g = GpuSystem(sysm, precision)
    g.set_param("taylor_kernel", kernel)
    g.set_state(zu)
    g.set_vloc(vloc)
    g.update_projector(kAc)
    return g


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_resident_step_matches_oracle(case, precision):
    _, sysm, kAc, vloc, zu = case
    dt = 0.08
    _, zproj = O.update_projector(sysm, kAc)
    z_ref = zu if precision == "c128" else zu.astype(np.complex64).astype(np.complex128)
    with _gpu(sysm, kAc, vloc, zu, precision, 2) as g:
        g.set_param("launches", 0)
        g.hamiltonian(dt)
        assert g.get_param("launches") == 1  # the whole step is one kernel
        g.hamiltonian(dt)
        for _ in range(2):
            z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, dt, z_ref)
        assert rel(g.get_state(), z_ref) < 2 * TOL[precision]


def test_resident_and_pass_forms_agree(case):
    _, sysm, kAc, vloc, zu = case
    out = []
    for kernel in (1, 2):
        with _gpu(sysm, kAc, vloc, zu, "c128", kernel) as g:
            g.hamiltonian(0.05)
            out.append(g.get_state())
    assert rel(out[1], out[0]) < 1e-13


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_flag_current_matches_oracle(case, precision, kernel):
    """hamiltonian(dt, flag_current) computes the current's stencil sums of the
    new orbitals with the step; current_RT at the new k+A then uses them."""
    _, sysm, kAc, vloc, zu = case
    kcur = kAc + np.array([0.0, 2e-3, 0.0])[:, None]
    with _gpu(sysm, kAc, vloc, zu, precision, kernel) as g:
        g.hamiltonian(0.08, flag_current=True)
        z = g.get_state()
        j = g.current_RT(kcur)
        assert rel(j, O.current(sysm, kcur, z)) < 1e-12
        # a step without the flag: the current is computed from the orbitals again
        g.hamiltonian(0.08)
        z = g.get_state()
        assert rel(g.current_RT(kcur), O.current(sysm, kcur, z)) < 1e-12


@pytest.mark.parametrize("nb", [1, 3, 5, 7])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_resident_ragged_band_groups(cuda_lib, precision, nb):
    """Band counts that leave the last band group of a k-point partly empty
    (complex(4) groups of 4 bands, complex(8) of 2 on 16x16 planes), with the
    current computed in the step."""
    sysm, kAc, vloc, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (3, 1, 1), nb, A=(0.0, 0.0, 1e-2))
    dt = 0.08
    _, zproj = O.update_projector(sysm, kAc)
    z_ref = zu if precision == "c128" else zu.astype(np.complex64).astype(np.complex128)
    z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, dt, z_ref)
    with _gpu(sysm, kAc, vloc, zu, precision, 2) as g:
        g.hamiltonian(dt, flag_current=True)
        z = g.get_state()
        assert rel(z, z_ref) < TOL[precision]
        kcur = kAc + np.array([1e-3, 0.0, 0.0])[:, None]
        assert rel(g.current_RT(kcur), O.current(sysm, kcur, z)) < 1e-12
