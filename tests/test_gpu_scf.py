"""Self-consistent local potential (Hartree + PZ LDA) on the GPU against the CPU
oracle (oracle/scf_oracle.py), a self-consistent ground state, and the FP32
path's J(t) under a self-consistent potential.

Tolerances: Vloc and the energies 1e-12 relative (FP64 FFTs); J(t) 1e-5
relative to max |J| (the FP32+FP64-reduce target)."""
import numpy as np
import pytest

from oracle import scf_oracle as X
from salmon_b200 import drive, system as S

pytestmark = pytest.mark.gpu

SI8 = dict(ncell=(1, 1, 1), grid=(16, 16, 16), nkgrid=(2, 2, 2), Nb=12, Nocc=8)  # 4 empty buffer bands


def _gpu(sysm, kAc, vpsl, precision="c128"):
    from salmon_b200.rt import GpuSystem
    g = GpuSystem(sysm, precision)
    g.set_vpsl(vpsl)
    g.set_vloc(vpsl)
    g.update_projector(kAc)
    return g


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 9, 12)])
def test_vloc_matches_oracle(cuda_lib, shape):
    if shape == (16, 16, 16):
        sysm, kAc, vpsl, zu = S.si_supercell_system(**SI8)
    else:
        sysm, kAc, vpsl, zu = S.small_system(*shape, nk=2, nb=3)
    rng = np.random.default_rng(8)
    rho = rng.uniform(1e-4, 0.3, sysm.NL)
    g = _gpu(sysm, kAc, vpsl)
    eh, exc = g.update_vloc(rho)
    v = g.get_vloc()
    want, (eh0, exc0) = X.vloc(rho, vpsl, shape, sysm.aL, sysm.Hxyz)
    assert np.abs(v - want).max() <= 1e-12 * np.abs(want).max()
    assert abs(eh - eh0) <= 1e-12 * abs(eh0) and abs(exc - exc0) <= 1e-12 * abs(exc0)
    # the resident orbitals' density is used when no rho is given
    g.set_state(zu[:, :sysm.NBoccmax])
    g.update_vloc()
    v1 = g.get_vloc()
    want1, _ = X.vloc(g.psi_rho_RT(), vpsl, shape, sysm.aL, sysm.Hxyz)
    assert np.abs(v1 - want1).max() <= 1e-12 * np.abs(want1).max()
    g.close()


@pytest.fixture(scope="module")
def scf_ground(cuda_lib):
    sysm, kAc, vpsl, zu = S.si_supercell_system(**SI8)
    kAc0 = np.ascontiguousarray(sysm.kAc0)
    g = _gpu(sysm, kAc0, vpsl)
    g.gs_set_state(zu)
    g.set_state(zu[:, :sysm.NBoccmax])
    g.update_vloc()
    g.set_cg_preconditioner("tpa")
    esp, hist = drive.ground_state_scf(g, n_iter=60, ncg=4, mix=0.2)
    zgs = g.gs_get_state()
    g.close()
    return sysm, kAc0, vpsl, zgs, hist


def test_scf_ground_state_converges(scf_ground):
    *_, hist = scf_ground
    print("scf", hist[::10], hist[-1])
    assert hist[-1][2] < 1e-3 * hist[1][2]    # density change between iterations falls 1000x
    assert hist[-1][1] < 1e-4                  # and the band residuals with it


def test_current_fp32_matches_fp64_with_scf_potential(scf_ground):
    from salmon_b200.rt import GpuSystem
    sysm, kAc0, vpsl, zgs, _ = scf_ground
    Nt, dt = 200, 0.08
    Ac = drive.init_Ac(Nt, dt, "impulse", epdir=(1.0, 0.0, 0.0), e_impulse=1e-2)
    out = {}
    for prec in ("c128", "c64"):
        with GpuSystem(sysm, "c128") as g:
            g.set_vloc(vpsl)
            g.update_projector(kAc0)
            g.gs_set_state(zgs)
            g.gs_to_rt()
            if prec == "c64":
                g.set_precision("c64")
            out[prec] = drive.rt_propagate(g, sysm, kAc0, vpsl, Ac, dt, Nt, energy_every=50, scf=True)
    (j64, e64), (j32, e32) = out["c128"], out["c64"]
    print("J error", drive.j_error(j64, j32), "E", e64[0], e64[Nt], e32[Nt])
    assert drive.j_error(j64, j32) < 1e-5
    for t in e64:
        assert abs((e32[t] - e32[0]) - (e64[t] - e64[0])) <= 1e-6
