"""Parity with the CPU oracle at the band counts and shapes the workloads run:
the tilings that small cases never reach.

  32^3, one k-point x 32 bands    one band group of the KB tile kernel (the
                                  hpsi/Taylor microbench's per-k-point tiling)
  32^3, one k-point x 128 bands   the Si64 supercell with the physical Si
                                  pseudopotential: four band groups; each KB
                                  kernel form (auto, tile, band quad, split tile)
  48^3, one k-point x 432 bands   the Si216 shape: the y-block stencil pass with
                                  fourteen band groups
  batched Si8 + Si16 + Si64       one CUDA-graph replay of the three systems,
                                  each compared with the oracle

Tolerances (max |gpu - oracle| / max |oracle|): complex(8) 1e-12; complex(4)
2e-6 per Taylor step; FP64 reductions of the propagated orbitals 1e-12 against
the oracle run on the same orbitals.
"""
import os

import numpy as np
import pytest

from _helpers import GOLDEN, rel
from oracle import oracle as O
from salmon_b200 import pseudo as P, system as S

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-12, "c64": 2e-6}


def c64_round(z):
    return z.astype(np.complex64).astype(np.complex128)


def _gpu(sysm, kAc, vloc, zu, precision, kb_kernel=0):
    from salmon_b200.rt import GpuSystem
    g = GpuSystem(sysm, precision)
    g.set_param("kb_kernel", kb_kernel)
    g.set_state(zu)
    g.set_vloc(vloc)
    g.update_projector(kAc)
    return g


def _steps_and_reductions(sysm, kAc, vloc, zu, precision, nsteps=1, kb_kernel=0):
    dt = 0.08
    _, zproj = O.update_projector(sysm, kAc)
    z_ref = zu if precision == "c128" else c64_round(zu)
    with _gpu(sysm, kAc, vloc, zu, precision, kb_kernel) as g:
        for _ in range(nsteps):
            g.hamiltonian(dt)
        got = g.get_state()
        for _ in range(nsteps):
            z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, dt, z_ref)
        err = rel(got, z_ref)
        assert err < TOL[precision] * nsteps, err
        # FP64 reductions of the propagated orbitals against the oracle on the same orbitals
        kcur = kAc + np.array([0.0, 0.0, 1e-3])[:, None]
        assert rel(g.psi_rho_RT(), O.psi_rho(sysm, got)) < 1e-12
        assert rel(g.current_RT(kcur), O.current(sysm, kcur, got)) < 1e-12


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_microbench_32_one_k_32_bands(cuda_lib, precision):
    sysm, kAc, vloc, zu = S.microbench_system(32, nk_limit=1, Nb=32)
    _steps_and_reductions(sysm, kAc, vloc, zu, precision, nsteps=2)


def _si64_pp():
    tabs = P.prepare(P.from_npz(os.path.join(GOLDEN, "si_rps_ky.npz"), lloc=2))
    sysm, kAc0, vpsl, zu = S.si_pp_system(tabs, ncell=(2, 2, 2), grid=(32, 32, 32), nkgrid=(1, 1, 1), NB=128,
                                          Nocc=128)
    kAc = np.ascontiguousarray(kAc0 + np.array([0.0, 0.0, 1e-2])[:, None])
    return sysm, kAc, vpsl, zu


@pytest.mark.parametrize("kb_kernel", [0, 1, 2, 3])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_si64_pseudopotential_128_bands(cuda_lib, precision, kb_kernel):
    sysm, kAc, vloc, zu = _si64_pp()
    assert sysm.NBoccmax == 128 and sysm.nk_local == 1
    _steps_and_reductions(sysm, kAc, vloc, zu, precision, nsteps=1, kb_kernel=kb_kernel)


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_wide_48_one_k_432_bands(cuda_lib, precision):
    sysm, kAc, vloc, zu = S.microbench_system(48, nk_limit=1, Nb=432)
    _steps_and_reductions(sysm, kAc, vloc, zu, precision, nsteps=1)


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batched_systems_against_oracle(cuda_lib, precision):
    """The three batched systems (Si8 16^3, Si16 16x16x32, Si64 32^3 with 128
    bands) at reduced k-point counts, advanced together by one graph replay of
    two steps each, each compared with the oracle's two steps."""
    from salmon_b200.rt import GpuBatch, GpuSystem
    shapes = [((1, 1, 1), (16, 16, 16), (2, 1, 1), 16), ((1, 1, 2), (16, 16, 32), (1, 1, 1), 32),
              ((2, 2, 2), (32, 32, 32), (1, 1, 1), 128)]
    dts = [0.08, 0.05, 0.04]
    nsteps = 2
    items = [S.si_supercell_system(nc, grid, nkg, nb, A=(0.0, 1e-2, 0.0)) for nc, grid, nkg, nb in shapes]
    gs = []
    try:
        for sysm, kAc, vloc, zu in items:
            g = GpuSystem(sysm, precision)
            g.set_state(zu)
            g.set_vloc(vloc)
            g.update_projector(kAc)
            gs.append(g)
        with GpuBatch(gs) as b:
            b.step(dts, nsteps)   # later calls on each handle are ordered after the replay
        for (sysm, kAc, vloc, zu), g, dt in zip(items, gs, dts):
            _, zproj = O.update_projector(sysm, kAc)
            z_ref = zu if precision == "c128" else c64_round(zu)
            for _ in range(nsteps):
                z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, dt, z_ref)
            err = rel(g.get_state(), z_ref)
            assert err < TOL[precision] * nsteps, (sysm.NLx, sysm.NLy, sysm.NLz, err)
    finally:
        for g in gs:
            g.close()
