"""Batched systems (one CUDA-graph replay advances every system) and the
autotuner, against the same systems stepped one call at a time.

The graph replays exactly the kernels of sgpu_hamiltonian, so the states agree
to 1e-13 relative (complex(8)) and 1e-6 (complex(4)); the autotuner only
changes launch shapes and the order of the projection sums: 1e-12 / 2e-6."""
import numpy as np
import pytest

from salmon_b200 import system as S

pytestmark = pytest.mark.gpu
TOL = {"c128": 1e-13, "c64": 1e-6}


def _systems():
    out = []
    sysm, kAc, vloc, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (2, 2, 2), 8)
    out.append((sysm, kAc, vloc, zu))
    sysm, kAc, vloc, zu = S.si_supercell_system((1, 1, 2), (16, 16, 32), (2, 2, 1), 12)
    out.append((sysm, kAc, vloc, zu))
    out.append(S.small_system(8, 9, 10, nk=3, nb=5))   # overlapping spheres, odd sizes
    return out


def _open(items, precision):
    from salmon_b200.rt import GpuSystem
    gs = []
    for sysm, kAc, vloc, zu in items:
        g = GpuSystem(sysm, precision)
        g.set_param("kb_kernel", 1)  # the tile KB kernel: a fixed launch count per stage
        g.set_state(zu)
        g.set_vloc(vloc)
        g.update_projector(kAc)
        gs.append(g)
    return gs


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batch_graph_matches_sequential_steps(cuda_lib, precision):
    from salmon_b200.rt import GpuBatch
    items = _systems()
    dts = [0.08, 0.05, 0.02]
    nsteps = 3
    ref = _open(items, precision)
    for g, dt in zip(ref, dts):
        for _ in range(2 * nsteps):
            g.hamiltonian(dt)
    want = [g.get_state() for g in ref]
    for g in ref:
        g.close()
    gs = _open(items, precision)
    with GpuBatch(gs) as b:
        for g in gs:
            g.set_param("launches", 0)
        b.step(dts, nsteps)      # captures, then replays
        b.step(dts, nsteps)      # replays the same graph
        counts = [g.get_param("launches") for g in gs]
        got = [g.get_state() for g in gs]
    for g in gs:
        g.close()
    for w, x in zip(want, got):
        assert _rel(x, w) <= TOL[precision]
    # 16x16 planes take the shared-memory resident step: one kernel per Taylor
    # step; the other systems the stencil passes: 2 kernels per stage (KB term,
    # stencil pass) +1 for the entry-wise KB field where spheres overlap, 4 stages
    # per step; 2 x nsteps steps
    assert counts[0] == 2 * nsteps
    assert counts[1] == 2 * nsteps * 4 * 2
    assert counts[2] == 2 * nsteps * 4 * 3


def test_batch_recaptures_on_new_dt(cuda_lib):
    from salmon_b200.rt import GpuBatch
    items = _systems()[:2]
    ref = _open(items, "c128")
    for g in ref:
        g.hamiltonian(0.08)
        g.hamiltonian(0.04)
    want = [g.get_state() for g in ref]
    for g in ref:
        g.close()
    gs = _open(items, "c128")
    with GpuBatch(gs) as b:
        b.step([0.08, 0.08], 1)
        b.step([0.04, 0.04], 1)
        got = [g.get_state() for g in gs]
    for g in gs:
        g.close()
    for w, x in zip(want, got):
        assert _rel(x, w) <= TOL["c128"]


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_autotune_keeps_results(cuda_lib, precision):
    sysm, kAc, vloc, zu = S.si_supercell_system((1, 1, 2), (16, 16, 32), (2, 2, 1), 12)
    (g0,) = _open([(sysm, kAc, vloc, zu)], precision)
    g0.hamiltonian(0.08)
    want = g0.get_state()
    g0.close()
    (g,) = _open([(sysm, kAc, vloc, zu)], precision)
    nslab, split, ms = g.autotune(reps=2)
    assert nslab in (1, 2, 4) and split in (0, 1, 2, 4, 8) and ms > 0
    assert g.get_param("nslab") == nslab
    if split == 0:  # the band-group tile kernel
        assert g.get_param("kb_kernel") == 1
    else:
        assert g.get_param("kb_kernel") == 2 and g.get_param("uvpsi_split") == split
    np.testing.assert_array_equal(g.get_state(), zu.astype(np.complex64 if precision == "c64" else np.complex128)
                                  .astype(np.complex128))
    g.hamiltonian(0.08)
    got = g.get_state()
    g.close()
    assert _rel(got, want) <= (1e-12 if precision == "c128" else 2e-6)
