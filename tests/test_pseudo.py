"""Pseudopotential ingest (KY format), Broyden mixing and the analytic rows of
SALMON's bulk-Si testsuite verification tables, on the CPU.

Fixtures: tests/golden/si_rps_ky.npz (testsuites/pseudo/Si_rps.dat as parsed) and
tests/golden/testsuite_si.json (inputs and verification tables of
testsuites/001_bulk_gs and 002_bulk_rt), made by tests/golden/make_testsuite_golden.py.
"""
import json
import os

import numpy as np
import pytest

from _helpers import GOLDEN
from salmon_b200 import broyden, drive, pseudo as P, system as S



def _si():
    return P.from_npz(os.path.join(GOLDEN, "si_rps_ky.npz"), lloc=2)


def _suite():
    with open(os.path.join(GOLDEN, "testsuite_si.json")) as f:
        return json.load(f)


def test_fixture_matches_reader():
    from oracle import oracle as O
    root = O.ref_root()
    if root is None:
        pytest.skip("reference tree not present (set REF_ROOT)")
    a = P.read_ps_ky(os.path.join(root, "testsuites", "pseudo", "Si_rps.dat"), lloc=2)
    b = _si()
    assert a.mr == b.mr and a.zps == b.zps == 4 and a.mlps == b.mlps == 2
    assert np.array_equal(a.vpp, b.vpp) and np.array_equal(a.upp, b.upp) and np.array_equal(a.rrc, b.rrc)


def test_tables_si():
    t = P.prepare(_si())
    # d channel is the local one (lloc_ps = 2): no projector; s and p are
    assert list(t.inorm) == [1, 1, 0]
    assert t.anorm[2] == 0.0 and t.anorm[0] > 0 and t.anorm[1] > 0
    # Rps = 1.2 A; the first radial point beyond it (1-based) and the table rows up to it
    assert abs(t.pp.rps - 1.2 / P.AU_LENGTH_AA) < 1e-15
    assert t.pp.nrps == 122 and t.radnl.size == 122 and t.vloctbl.size == 122
    assert np.all(t.radnl[:-1] <= t.pp.rps) and t.radnl[-1] > t.pp.rps
    # the local channel approaches -Zps/r at the cut-off
    assert abs(t.vloctbl[-1] * t.radnl[-1] + 4.0) < 0.05


def test_spline_is_natural_cubic():
    from scipy.interpolate import CubicSpline
    t = P.prepare(_si())
    for l in (0, 1):
        a, b, c, d = P.spline(t.radnl, t.udvtbl[:, l])
        cs = CubicSpline(t.radnl, t.udvtbl[:, l], bc_type="natural")
        scale = np.abs(t.udvtbl[:, l]).max()
        for mine, ref in ((a, cs.c[0]), (b, cs.c[1]), (c, cs.c[2]), (d, cs.c[3])):
            assert np.abs(mine - ref).max() <= 1e-9 * scale / t.pp.step ** 3


def test_kb_tables_and_vpsl_si8():
    t = P.prepare(_si())
    sysm, kAc0, vpsl, zu = S.si_pp_system(t, with_orbitals=False)
    assert list(sysm.Mps) == [27] * 8 and sysm.Nlma == 32
    assert list(sysm.iuV[:4]) == [1, 1, 1, 1] and list(sysm.a_tbl[:8]) == [1, 1, 1, 1, 2, 2, 2, 2]
    # projectors of different m on the same atom are orthogonal on a symmetric sphere
    u = sysm.uV[:4, :27]
    gram = u @ u.T
    assert np.abs(gram - np.diag(np.diag(gram))).max() < 1e-12 * np.abs(gram).max()
    # the FFT evaluation of Vpsl equals the direct G sum of calc_vpsl
    gx, gy, gz, m0 = P.g_vectors(8, 8, 8, sysm.aL)
    g2 = gx * gx + gy * gy + gz * gz
    dv = P.calc_vloc(t, np.sqrt(g2))
    coul = np.zeros_like(g2)
    nz = np.arange(g2.size) != m0
    coul[nz] = 4 * np.pi / g2[nz] * 4
    vion = sum((dv - coul) * np.exp(-1j * (gx * R[0] + gy * R[1] + gz * R[2])) for R in sysm.Rion) / sysm.aLxyz
    lx, ly, lz = sysm.grid_coords()
    h = sysm.H
    phase = np.exp(1j * (np.outer(lx * h[0], gx) + np.outer(ly * h[1], gy) + np.outer(lz * h[2], gz)))
    direct = np.real(phase @ vion)
    assert np.abs(direct - vpsl).max() <= 1e-12 * np.abs(direct).max()


def test_broyden_first_step_and_convergence():
    """On a linear fixed-point problem rho_out = J rho + c with slow modes
    (eigenvalues of J up to 0.97), the first step is linear mixing and 20
    Broyden steps beat 20 linear-mixing steps by more than 50x."""
    rng = np.random.default_rng(3)
    n = 64
    q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    jac = q @ np.diag(rng.uniform(0.5, 0.97, n)) @ q.T
    fixed = rng.uniform(1.0, 2.0, n)                             # positive, like a density
    c = fixed - jac @ fixed
    x0 = np.full(n, 1.5)
    m = broyden.Broyden()
    m.start(x0)
    x = m.mix(jac @ x0 + c)
    assert np.allclose(x, x0 + 0.75 * (jac @ x0 + c - x0))       # first iteration is linear mixing
    for _ in range(19):
        x = m.mix(jac @ x + c)
    lin = x0.copy()
    for _ in range(20):
        lin = lin + 0.75 * (jac @ lin + c - lin)
    assert np.abs(x - fixed).max() < 2e-2 * np.abs(lin - fixed).max()


def _rows(table, fname):
    return [r for r in table if r["file"] == fname]


def test_k_points_and_occupations_match_001():
    suite = _suite()
    bl = 2 * np.pi / np.asarray(suite["inputs"]["al"])
    k = S.uniform_k_grid(4, 4, 4, bl)
    for r in _rows(suite["001_bulk_gs"], "Si_k.data"):
        ik, col = r["row"], r["col"]
        got = 1.0 if col == 4 else k[col - 1, ik] / bl[col - 1]      # kw = 1 (Sym = 1)
        assert abs(got - r["value"]) <= r["tol"], r["label"]
    t = P.prepare(_si())
    sysm, _, _, _ = S.si_pp_system(t, with_orbitals=False)
    for r in _rows(suite["001_bulk_gs"], "Si_eigen.data"):
        if r["col"] != 3:
            continue
        ik, ib = divmod(r["row"], 32)
        assert abs(sysm.occ[ik, ib] * sysm.NK - r["value"]) <= r["tol"], r["label"]


def test_pulse_matches_002():
    """Ac_tot and E_tot rows of Si_rt.data: the Acos2 pulse of init_Ac with E = -dA/dt
    by the central difference of control_sc.f90:218-220."""
    suite = _suite()
    inp = suite["inputs"]
    dt, nt = inp["dt"], inp["nt"]
    Ac = drive.init_Ac(nt + 1, dt, "Acos2", epdir=inp["epdir_re1"], rlaser_int_wcm2=inp["rlaser_int_wcm2_1"],
                       omega=inp["omega1"], pulse_tw=inp["pulse_tw1"])
    for r in _rows(suite["002_bulk_rt"], "Si_rt.data"):
        it, col = r["row"], r["col"]
        if col == 9:
            got = Ac[it + 1, 2]
        elif col == 12:
            got = -(Ac[it + 2, 2] - Ac[it, 2]) / (2 * dt)
        else:
            continue
        assert abs(got - r["value"]) <= r["tol"], (r["label"], got)


def test_ewald_energy_converges_and_is_independent_of_the_split():
    """With a G set large enough (24^3) the Ewald sum does not depend on the
    splitting parameter; diamond Si at a = 10.26 bohr gives about -8.40 Ry per atom.
    On the 8^3 grid's G set the reciprocal sum is truncated, as in the reference."""
    aL = np.array([10.26] * 3)
    R = S.DIAMOND_RED * aL
    e3 = P.ewald_energy(R, 4.0, aL, (24, 24, 24), a_ewald=0.3)
    e5 = P.ewald_energy(R, 4.0, aL, (24, 24, 24), a_ewald=0.5)
    assert abs(e3 - e5) < 1e-9 * abs(e5)
    assert -8.45 < 2 * e5 / 8 < -8.35
    assert abs(P.ewald_energy(R, 4.0, aL, (8, 8, 8)) - e5) > 0.1


def test_gs_wfn_files_round_trip_and_layout(tmp_path):
    from salmon_b200 import wfn_io
    rng = np.random.default_rng(5)
    NK, NB, NL = 3, 4, 10
    zu = rng.standard_normal((NK, NB, NL)) + 1j * rng.standard_normal((NK, NB, NL))
    occ = rng.uniform(0, 1, (NK, NB))
    wfn_io.write_gs_wfn_k(str(tmp_path), zu, occ)
    z2, o2 = wfn_io.read_gs_wfn_k(str(tmp_path), NK, NB, NL)
    assert np.array_equal(z2, zu) and np.array_equal(o2, occ)
    raw = (tmp_path / "gs_wfn_k" / "wfn_gs_k0000002.wfn").read_bytes()
    n = NB * NL * 16
    assert len(raw) == n + 8
    assert int.from_bytes(raw[:4], "little") == n and int.from_bytes(raw[-4:], "little") == n
    # column-major zu_GS(NL, NB): the first NL values are band 1 of k-point 2
    first = np.frombuffer(raw[4:4 + 16 * NL], dtype="<c16")
    assert np.array_equal(first, zu[1, 0])
    occ_raw = (tmp_path / "gs_wfn_k" / "occupation").read_bytes()
    assert np.array_equal(np.frombuffer(occ_raw[4:-4], dtype="<f8")[:NB], occ[0])   # occ(1:NB, 1)
    # a damaged record is refused
    (tmp_path / "gs_wfn_k" / "wfn_gs_k0000003.wfn").write_bytes(raw[:-2])
    with pytest.raises(ValueError):
        wfn_io.read_gs_wfn_k(str(tmp_path), NK, NB, NL)


def test_d_projectors_with_s_local():
    """With the s channel local (lloc = 0) the p and d channels carry projectors:
    3 + 5 per atom.  The atoms sit on grid points of the 8^3 grid, so each sphere
    is cubic-symmetric and projectors of different (l, m) are orthogonal on it; the
    d functions follow the Ylm table (e.g. r^2 Y_20 ~ (3z^2 - r^2)/2)."""
    t = P.prepare(P.from_npz(os.path.join(GOLDEN, "si_rps_ky.npz"), lloc=0))
    assert list(t.inorm[1:] != 0) == [True, True] and t.inorm[0] == 0
    sysm, kAc0, vpsl, zu = S.si_pp_system(t, with_orbitals=False)
    assert sysm.Nlma == 8 * 8 and list(sysm.a_tbl[:9]) == [1] * 8 + [2]
    m = int(sysm.Mps[0])
    u = sysm.uV[:8, :m]
    gram = u @ u.T
    assert np.abs(gram - np.diag(np.diag(gram))).max() < 1e-12 * np.abs(gram).max()
    # r^2 Y_20 ~ (3z^2 - r^2)/2 times a radial factor: zero where 3z^2 = r^2, and the
    # ratio to (3z^2 - r^2) depends on r only
    _, _, _, _, _, dist = S.calc_jxyz(8, 8, 8, sysm.aL, sysm.Rion, t.pp.rps)
    x, y, z = dist[0, :m, 0], dist[0, :m, 1], dist[0, :m, 2]
    d0 = u[3 + 2]                                            # l = 2, m = 0 (after the three p)
    ang = 3 * z * z - (x * x + y * y + z * z)
    scale = np.abs(d0).max()
    zero = np.abs(ang) < 1e-9
    assert zero.any() and np.abs(d0[zero]).max() < 1e-12 * scale
    r = np.round(np.sqrt(x * x + y * y + z * z), 9)
    for rr in np.unique(r[~zero]):
        sel = (~zero) & (r == rr)
        ratio = d0[sel] / ang[sel]
        assert np.abs(ratio - ratio[0]).max() <= 1e-12 * np.abs(ratio).max()
