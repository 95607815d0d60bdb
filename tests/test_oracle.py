"""Pins the CPU oracle (oracle/) before anything is checked against it.

The oracle is pinned by (1) golden vectors produced by SALMON's own compiled
AVX kernels (tests/golden, made by tests/golden/make_golden.py), (2) the same
kernels run live when oracle/_ref is built, and (3) known answers of the
discretised operator: the closed-form Nd=4 coefficients, the plane-wave symbol,
Hermiticity and the O(dt^5) local error of the 4th-order Taylor step."""
import numpy as np
import pytest

from _helpers import coefs, grid_system, load_golden, rel, system_from_arrays
from oracle import oracle as O
from salmon_b200 import system as S


def test_fd_coef_known_answers():
    lap, nab = O.fd_coef(4)
    exact_lap = [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560]
    exact_nab = [4 / 5, -1 / 5, 4 / 105, -1 / 280]
    np.testing.assert_allclose(lap[4:], exact_lap, rtol=1e-15, atol=1e-16)
    np.testing.assert_allclose(lap[:4][::-1], exact_lap[1:], rtol=1e-15)
    np.testing.assert_allclose(nab[5:], exact_nab, rtol=1e-15)
    np.testing.assert_allclose(nab[:4][::-1], -np.array(exact_nab), rtol=1e-15)
    lp, nb = S.fd_coef(4)  # the host-side copy used by the C descriptor
    np.testing.assert_array_equal(lp, lap)
    np.testing.assert_array_equal(nb, nab)


@pytest.mark.parametrize("name", ["ref_stencil_8x10x12.npz", "ref_stencil_16x16x16.npz"])
def test_stencil_matches_reference_avx_golden(name):
    g = load_golden(name)
    sysm = grid_system(tuple(int(v) for v in g["shape"]))
    F = O.stencil(sysm, float(g["A"]), g["B"], g["C"], g["D"], g["E"])
    assert rel(F, g["F"]) < 1e-14


def test_current_stencil_golden():
    g = load_golden("ref_current_stencil.npz")
    sysm = grid_system(tuple(int(v) for v in g["shape"]), nk=1, nb=1)
    # current() with occ=1, kAc=0 and no projectors reduces to the stencil sums times Hxyz/aLxyz
    zu = g["E"].reshape(1, 1, -1)
    jav = O.current(sysm, np.zeros((3, 1)), zu)
    expect = g["FGH"] * sysm.Hxyz / sysm.aLxyz
    assert rel(jav, expect) < 1e-13


def test_total_energy_stencil_golden():
    g = load_golden("ref_total_energy_stencil.npz")
    sysm = grid_system(tuple(int(v) for v in g["shape"]))
    # Ekin with occ=1 = Re(tpsum) Hxyz + |k|^2/2; use k=0 so nabt=0: compare with D=0 reference value
    F = g["F"][0]
    # rebuild k from D = k_d nab_d
    ln = sysm.lap_nab()
    k = np.array([g["D"][0] / ln["nabx"][1], g["D"][4] / ln["naby"][1], g["D"][8] / ln["nabz"][1]])
    ek, en = O.energy_terms(sysm, k.reshape(3, 1), g["E"].reshape(1, 1, -1))
    assert en == 0.0
    assert abs(ek - (F.real * sysm.Hxyz + k @ k / 2)) < 1e-13 * abs(ek)


def test_taylor_step_golden():
    g = load_golden("ref_taylor_step.npz")
    sysm = system_from_arrays(g)
    _, zproj = O.update_projector(sysm, g["kAc"])
    z1 = O.hamiltonian(sysm, g["kAc"], g["vloc"], zproj, float(g["dt"]), g["zu"])
    assert rel(z1, g["zu_next"]) < 1e-14


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref (reference AVX build) not present")
@pytest.mark.parametrize("shape", [(8, 10, 12), (12, 8, 16), (16, 16, 16), (20, 20, 20)])
def test_stencil_matches_reference_avx_live(shape):
    sysm, kAc, vloc, zu = S.small_system(*shape, nk=1, nb=1, seed=sum(shape))
    lapt, _, nabt, A = coefs(sysm, kAc[:, 0])
    F1 = O.stencil(sysm, A, vloc, lapt, nabt, zu[0, 0])
    F2 = O.ref_stencil(sysm, A, vloc, lapt, nabt, zu[0, 0])
    assert rel(F1, F2) < 1e-14


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref (reference AVX build) not present")
def test_taylor_step_matches_reference_avx_live():
    sysm, kAc, vloc, zu = S.small_system(10, 8, 14, nk=2, nb=3, seed=5)
    _, zproj = O.update_projector(sysm, kAc)
    z1 = O.hamiltonian(sysm, kAc, vloc, zproj, 0.04, zu)
    za = O.aligned_state(zu)
    O.ref_hamiltonian(sysm, kAc, vloc, zproj, 0.04, za)
    assert rel(z1, za) < 1e-14


def test_plane_wave_symbol():
    """For psi = exp(i G.r) the stencil returns (FD symbol of |G+k|^2/2 + V0) psi."""
    shape = (8, 10, 12)
    sysm = grid_system(shape, aL=(6.0, 6.5, 7.0))
    h = sysm.H
    ix, iy, iz = sysm.grid_coords()
    r = np.stack([ix * h[0], iy * h[1], iz * h[2]], axis=1)
    G = 2 * np.pi * np.array([1, -2, 3]) / sysm.aL
    k = np.array([0.11, -0.07, 0.05])
    psi = np.exp(1j * r @ G)
    V0 = 0.37
    lapt, _, nabt, A = coefs(sysm, k)
    F = O.stencil(sysm, A, np.full(sysm.NL, V0), lapt, nabt, psi)
    lap, nab = S.fd_coef()
    sym = V0 + 0.5 * (k @ k)
    for d in range(3):
        gh = G[d] * h[d]
        sym += -0.5 * (lap[4] + 2 * sum(lap[4 + n] * np.cos(n * gh) for n in range(1, 5))) / h[d] ** 2
        sym += k[d] * 2 * sum(nab[4 + n] * np.sin(n * gh) for n in range(1, 5)) / h[d]
    assert rel(F, sym * psi) < 1e-13


def test_hpsi_hermitian():
    sysm, kAc, vloc, zu = S.small_system(8, 10, 12, nk=2, nb=2, seed=3)
    _, zproj = O.update_projector(sysm, kAc)
    a, b = zu[1, 0], zu[1, 1]
    ha = O.hpsi(sysm, kAc, vloc, zproj, 2, a)
    hb = O.hpsi(sysm, kAc, vloc, zproj, 2, b)
    lhs = np.vdot(b, ha)
    rhs = np.conj(np.vdot(a, hb))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_taylor_local_error_is_fifth_order():
    """||U_taylor(dt) psi - exp(-iH dt) psi|| scales as dt^5 (smooth orbitals, fixed H)."""
    sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=1, nb=1, seed=4)
    _, zproj = O.update_projector(sysm, kAc)
    NL = sysm.NL
    Hm = np.empty((NL, NL), complex)
    eye = np.eye(NL)
    for j in range(NL):
        Hm[:, j] = O.hpsi(sysm, kAc, vloc, zproj, 1, eye[j])
    w, V = np.linalg.eigh(0.5 * (Hm + Hm.conj().T))
    # a smooth state: the lowest eigenvectors
    psi = V[:, :4] @ np.array([1, 0.5, 0.25, 0.125])
    errs = []
    for dt in (0.4, 0.2):
        exact = V @ (np.exp(-1j * w * dt) * (V.conj().T @ psi))
        z = O.hamiltonian(sysm, kAc, vloc, zproj, dt, psi.reshape(1, 1, -1))[0, 0]
        errs.append(np.linalg.norm(z - exact))
    assert 25 < errs[0] / errs[1] < 40


def test_cg_lowers_band_energies():
    sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=2, nb=3, seed=8)
    zg = O.gram_schmidt(sysm, zu)
    ov = np.einsum("kbi,kci->kbc", zg.conj(), zg) * sysm.Hxyz
    assert np.abs(ov - np.eye(3)[None]).max() < 1e-12
    z1, esp, its = O.cg(sysm, kAc, vloc, zg, 4)
    z2, esp2, _ = O.cg(sysm, kAc, vloc, z1, 4)
    assert esp2.sum() < esp.sum()
    assert its.min() >= 1
