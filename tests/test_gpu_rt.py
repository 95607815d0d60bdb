"""Real-time propagation on the GPU: complex(4) orbitals with FP64 reductions
against the complex(8) path, from a ground state, over many steps.

Tolerance on the macroscopic current: max_t |J_32(t) - J_64(t)| / max_t |J_64(t)|
<= 1e-5 (the target of the FP32+FP64-reduce path); the band-energy change
over the run agrees to 1e-6 Ha (a few FP32 ulps of the band energy itself)."""
import numpy as np
import pytest

from salmon_b200 import drive, system as S

pytestmark = pytest.mark.gpu


def _run(precision, sysm, kAc0, vloc, zgs, Nt, dt, Ac):
    from salmon_b200.rt import GpuSystem
    with GpuSystem(sysm, "c128") as g:
        g.set_vloc(vloc)
        g.update_projector(kAc0)
        g.gs_set_state(zgs)
        g.gs_to_rt()
        if precision == "c64":
            g.set_precision("c64")
        return drive.rt_propagate(g, sysm, kAc0, vloc, Ac, dt, Nt, energy_every=25)


@pytest.fixture(scope="module")
def ground(cuda_lib):
    from salmon_b200.rt import GpuSystem
    sysm, kAc, vloc, zu = S.microbench_system(16, nkgrid=(2, 2, 2), Nb=8)
    kAc0 = np.ascontiguousarray(sysm.kAc0)
    with GpuSystem(sysm) as g:
        g.set_vloc(vloc)
        g.update_projector(kAc0)
        g.gs_set_state(zu)
        esp, esp_var, hist = drive.ground_state(g, n_iter=40, ncg=4)
        zgs = g.gs_get_state()
    return sysm, kAc0, vloc, zgs, esp, esp_var, hist


def test_ground_state_converges(ground):
    sysm, kAc0, vloc, zgs, esp, esp_var, hist = ground
    assert np.all(np.diff(esp, axis=1) >= -1e-10)       # ascending, like zheev
    print("esp", esp[0], "history", hist[::5], hist[-1])
    sums = np.array([h[0] for h in hist])
    assert np.all(np.diff(sums) <= 1e-9 * np.abs(sums[1:]))   # variational: the band sum never rises
    assert hist[-1][1] < 0.05 * hist[0][1]                     # residuals fall by 20x
    ov = np.einsum("kbi,kci->kbc", zgs.conj(), zgs) * sysm.Hxyz
    assert np.abs(ov - np.eye(sysm.NB)[None]).max() < 1e-10


def test_current_fp32_matches_fp64(ground):
    sysm, kAc0, vloc, zgs = ground[:4]
    Nt, dt = 200, 0.08
    Ac = drive.init_Ac(Nt, dt, "impulse", epdir=(1.0, 0.0, 0.0), e_impulse=1e-2)
    j64, e64 = _run("c128", sysm, kAc0, vloc, zgs, Nt, dt, Ac)
    j32, e32 = _run("c64", sysm, kAc0, vloc, zgs, Nt, dt, Ac)
    print("J error", drive.j_error(j64, j32), "dynamic", drive.j_error_dynamic(j64, j32),
          "max|J|", np.abs(j64).max(), "E", {t: (e64[t], e32[t]) for t in (0, Nt)})
    assert drive.j_error(j64, j32) < 1e-5
    # the induced (time-dependent) current is resolved too
    assert drive.j_error_dynamic(j64, j32) < 1e-3
    for t in e64:
        de64 = e64[t] - e64[0]
        de32 = e32[t] - e32[0]
        assert abs(de32 - de64) <= 1e-6
