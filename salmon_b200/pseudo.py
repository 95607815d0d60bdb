"""Norm-conserving pseudopotentials for periodic systems: the radial tables of a
Yabana-Bertsch (KY, ``*_rps.dat``) file turned into the local potential Vpsl on
the grid and the Kleinman-Bylander tables (Mps, Jxyz, uV, iuV, a_tbl) that the
C ABI takes.

Reference routines restated here (paths relative to the SALMON source tree):
  read_ps_ky                  atom/pp/input_pp.f90:158-201
  anorm / inorm               atom/pp/input_pp.f90:64-90
  making_ps_without_masking   atom/pp/input_pp.f90:544-607 (udV and Vloc tables)
  spline                      atom/pp/prep_pp.f90:603-692 (natural cubic spline)
  calc_uv                     atom/pp/prep_pp.f90:420-601 (spline x Ylm on sphere points)
  set_lma_tbl                 atom/pp/prep_pp.f90:413-436 (projector numbering)
  Ylm                         atom/pp/Ylm_dYlm.f90:21-60 (l <= 2)
  calc_vloc                   atom/pp/prep_pp.f90:17-60  (dVloc(G) = FT of Vloc + Z/r)
  calc_vpsl                   atom/pp/prep_pp.f90:64-145 (Vpsl(r) from the structure factor)
  G vectors                   ARTED/preparation/init.f90:45-54
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

AU_LENGTH_AA = 0.52917721067   # io/inputoutput.f90:23
AU_ENERGY_EV = 27.21138505     # io/inputoutput.f90:22
EPS_NORM = 1e-10               # input_pp.f90:28 (Eps0)


@dataclass
class RadialPP:
    """One element's tables in atomic units.  Index i of rad / vpp / upp is the
    reference's 0-based file row i (rad(i+1) in the Fortran 1-based array)."""
    zps: int
    mlps: int
    lref: int
    step: float
    rrc: np.ndarray      # (mlps+1,) cut-off radii
    rad: np.ndarray      # (mr+2,)  rad[i] = i*step
    vpp: np.ndarray      # (mr+1, mlps+1)
    upp: np.ndarray      # (mr+1, mlps+1) raw radial functions
    mr: int

    @property
    def rps(self) -> float:
        return float(self.rrc.max())

    @property
    def nrps(self) -> int:
        """1-based index of the first radial point beyond rps (input_pp.f90:66-70)."""
        i = np.nonzero(self.rad[:self.mr + 1] > self.rps)[0]
        if i.size == 0:
            raise ValueError("NRps > Nrmax")
        return int(i[0]) + 1


def read_ps_ky(path: str, lloc: int, lmax_ps: int = -1) -> RadialPP:
    """Reads a KY ``*_rps.dat`` file: a header (Mr, step [A], Mlps, Zps), the
    cut-off radii, Mr+1 rows of (r, rho, V_l) and Mr+1 rows of (r, u_l), in
    Angstrom and eV; converts to atomic units (input_pp.f90:170-199)."""
    with open(path) as f:
        toks = f.read().split()
    pos = 0

    def take(n):
        nonlocal pos
        out = toks[pos:pos + n]
        pos += n
        return out

    mr, step, mlps, rzps = take(4)
    mr, step, mlps, rzps = int(mr), float(step), int(mlps), float(rzps)
    head = take(1 + mlps + 1)
    rrc = np.array([float(v) for v in head[1:]])
    vpp = np.zeros((mr + 1, mlps + 1))
    upp = np.zeros((mr + 1, mlps + 1))
    for i in range(mr + 1):
        row = take(2 + mlps + 1)
        vpp[i] = [float(v) for v in row[2:]]
    for i in range(mr + 1):
        row = take(1 + mlps + 1)
        upp[i] = [float(v) for v in row[1:]]
    return from_tables(mr, step, mlps, rzps, rrc, vpp, upp, lloc, lmax_ps)


def from_tables(mr, step, mlps, rzps, rrc, vpp, upp, lloc, lmax_ps=-1) -> RadialPP:
    """The unit conversion of read_ps_ky on already parsed file tables
    (Angstrom, eV, radial functions per sqrt(Angstrom))."""
    step = step / AU_LENGTH_AA
    rrc = np.asarray(rrc, dtype=np.float64) / AU_LENGTH_AA
    vpp = np.asarray(vpp, dtype=np.float64) / AU_ENERGY_EV
    upp = np.asarray(upp, dtype=np.float64) * np.sqrt(AU_LENGTH_AA)
    rad = np.arange(mr + 2, dtype=np.float64) * step
    if lmax_ps >= 0:
        mlps = lmax_ps
    return RadialPP(zps=int(rzps + 1e-10), mlps=mlps, lref=lloc, step=step, rrc=rrc[:mlps + 1], rad=rad,
                    vpp=vpp, upp=upp, mr=mr)


@dataclass
class PPTables:
    """Derived radial tables of one element (input_pp.f90:64-90, 544-607)."""
    pp: RadialPP
    anorm: np.ndarray    # (mlps+1,)
    inorm: np.ndarray    # (mlps+1,) in {-1, 0, +1}
    radnl: np.ndarray    # (nrps,) radii of the table rows
    udvtbl: np.ndarray   # (nrps, mlps+1)
    vloctbl: np.ndarray  # (nrps,)


def prepare(pp: RadialPP) -> PPTables:
    """anorm/inorm from the trapezoid rule over the whole radial grid with the raw
    u_l, then u_l * sqrt((2l+1)/4pi) / r^(l+1) and the tables
    udV_l = (V_l - V_lref) u_l / anorm_l and Vloc = V_lref on the first NRps rows."""
    mr, L = pp.mr, pp.mlps
    r1 = pp.rad[1:mr] - pp.rad[0:mr - 1]                        # rad(i+1) - rad(i), i = 1..mr-1
    anorm = np.zeros(L + 1)
    inorm = np.zeros(L + 1, np.int32)
    for l in range(L + 1):
        dv = pp.vpp[:, l] - pp.vpp[:, pp.lref]
        w = pp.upp[:, l] ** 2 * dv
        s = 0.0
        for i in range(1, mr):                                   # sequential, as the reference sums
            s += (w[i] + w[i - 1]) * r1[i - 1]
        s *= 0.5
        inorm[l] = 1
        if s < 0.0:
            s = -s
            inorm[l] = -1
        if abs(s) < EPS_NORM:
            inorm[l] = 0
        anorm[l] = np.sqrt(s)
    upp = pp.upp.copy()
    for l in range(L + 1):
        upp[1:mr + 1, l] = upp[1:mr + 1, l] * np.sqrt((2 * l + 1.0) / (4 * np.pi)) / pp.rad[1:mr + 1] ** (l + 1)
        upp[0, l] = upp[1, l]
    nrps = pp.nrps
    vloctbl = pp.vpp[:nrps, pp.lref].copy()
    udvtbl = np.zeros((nrps, L + 1))
    for l in range(L + 1):
        udvtbl[:, l] = (pp.vpp[:nrps, l] - pp.vpp[:nrps, pp.lref]) * upp[:nrps, l]
        if inorm[l] != 0:
            udvtbl[:, l] /= anorm[l]
    return PPTables(pp=pp, anorm=anorm, inorm=inorm, radnl=pp.rad[:nrps].copy(), udvtbl=udvtbl, vloctbl=vloctbl)


def spline(xn, yn):
    """Natural cubic spline through (xn, yn): per interval i the coefficients
    (a, b, c, d) of a*t^3 + b*t^2 + c*t + d, t = x - xn[i] (prep_pp.f90:603-692;
    the interior second derivatives solve the same tridiagonal system, here by
    the Thomas algorithm instead of an explicit inverse)."""
    xn = np.asarray(xn, dtype=np.float64)
    yn = np.asarray(yn, dtype=np.float64)
    n = xn.size
    dx = np.diff(xn)
    dy = np.diff(yn)
    m = n - 2
    v = 6.0 * (dy[1:] / dx[1:] - dy[:-1] / dx[:-1])            # v(1..m)
    diag = 2.0 * (dx[1:] + dx[:-1])
    lower = dx[:-1].copy()                                       # A(i, i-1) = dx(i-1)
    upper = dx[1:].copy()                                        # A(i, i+1) = dx(i)
    cp = np.zeros(m)
    dp = np.zeros(m)
    cp[0] = upper[0] / diag[0]
    dp[0] = v[0] / diag[0]
    for i in range(1, m):
        den = diag[i] - lower[i] * cp[i - 1]
        cp[i] = upper[i] / den if i < m - 1 else 0.0
        dp[i] = (v[i] - lower[i] * dp[i - 1]) / den
    u = np.zeros(m)
    u[m - 1] = dp[m - 1]
    for i in range(m - 2, -1, -1):
        u[i] = dp[i] - cp[i] * u[i + 1]
    uu = np.concatenate([[0.0], u, [0.0]])                       # second derivatives, natural ends
    b = 0.5 * uu[:-1]
    a = (uu[1:] - 2.0 * b) / (6.0 * dx)
    d = yn[:-1].copy()
    c = dy / dx - dx * (uu[1:] + 2.0 * uu[:-1]) / 6.0
    return a, b, c, d


def ylm(x, y, z, l, m):
    """r^l times the real spherical harmonic, scaled by sqrt(4pi/(2l+1))
    (Ylm_dYlm.f90:21-60), for l <= 2."""
    r2 = x * x + y * y + z * z
    table = {
        (0, 0): lambda: np.ones_like(x),
        (1, -1): lambda: -y, (1, 0): lambda: z, (1, 1): lambda: -x,
        (2, -2): lambda: np.sqrt(3.0) * x * y, (2, -1): lambda: -np.sqrt(3.0) * y * z,
        (2, 0): lambda: (3.0 * z * z - r2) / 2.0, (2, 1): lambda: -np.sqrt(3.0) * x * z,
        (2, 2): lambda: np.sqrt(3.0 / 4.0) * (x * x - y * y),
    }
    if (l, m) not in table:
        raise NotImplementedError(f"Ylm for l={l} (only l <= 2 is implemented)")
    return table[(l, m)]()


def kb_tables(tabs: PPTables, Mps, dist):
    """uV(Nlma, Nps), iuV(Nlma), a_tbl(Nlma) for atoms of one element on their
    sphere points (calc_uv, prep_pp.f90:538-583): the spline of udV_l at r times
    Ylm, projectors numbered atom by atom, l ascending, m = -l..l, channels with
    inorm = 0 skipped (set_lma_tbl)."""
    pp = tabs.pp
    a_, b_, c_, d_ = [], [], [], []
    for l in range(pp.mlps + 1):
        a, b, c, d = spline(tabs.radnl, tabs.udvtbl[:, l])
        a_.append(a); b_.append(b); c_.append(c); d_.append(d)
    ls = [l for l in range(pp.mlps + 1) if tabs.inorm[l] != 0]
    nproj = sum(2 * l + 1 for l in ls)
    NI, Nps = dist.shape[:2]
    uV = np.zeros((NI * nproj, Nps))
    iuV = np.zeros(NI * nproj, np.int32)
    a_tbl = np.zeros(NI * nproj, np.int32)
    nr = tabs.radnl.size
    for a in range(NI):
        m_a = int(Mps[a])
        x, y, z = dist[a, :m_a, 0], dist[a, :m_a, 1], dist[a, :m_a, 2]
        r = np.sqrt(x * x + y * y + z * z) + 1e-50
        # first table row with radnl > r, minus one (1-based intr of the reference)
        ir = np.array([int(np.nonzero(tabs.radnl > rr)[0][0]) + 1 if (tabs.radnl > rr).any() else nr + 1
                       for rr in r])
        intr = ir - 1
        if np.any(intr < 0) or np.any(intr >= nr):
            raise ValueError("sphere point beyond the radial table (bad intr)")
        k = intr - 1                                              # 0-based spline interval
        xx = r - tabs.radnl[intr - 1]
        lma = a * nproj
        for l in ls:
            uvr = a_[l][k] * xx ** 3 + b_[l][k] * xx ** 2 + c_[l][k] * xx + d_[l][k]
            for m in range(-l, l + 1):
                uV[lma, :m_a] = uvr * ylm(x, y, z, l, m)
                iuV[lma] = tabs.inorm[l]
                a_tbl[lma] = a + 1
                lma += 1
    return uV, iuV, a_tbl


def g_vectors(NLx, NLy, NLz, aL):
    """G = (ix bLx, iy bLy, iz bLz), ix in [-NLx/2, NLx-1-NLx/2] in the
    reference's loop order, and the index of G = 0 (init.f90:45-54)."""
    bl = 2 * np.pi / np.asarray(aL, dtype=np.float64)
    mx = np.arange(-(NLx // 2), NLx - NLx // 2)
    my = np.arange(-(NLy // 2), NLy - NLy // 2)
    mz = np.arange(-(NLz // 2), NLz - NLz // 2)
    gx, gy, gz = np.meshgrid(mx * bl[0], my * bl[1], mz * bl[2], indexing="ij")
    m0 = (NLx // 2) * NLy * NLz + (NLy // 2) * NLz + NLz // 2
    return gx.ravel(), gy.ravel(), gz.ravel(), m0


def calc_vloc(tabs: PPTables, g):
    """dVloc(G): the radial Fourier transform of Vloc(r) + Zps/r over the first
    NRps rows by the midpoint rule (prep_pp.f90:33-55).  g = |G| per G vector,
    with g = 0 at G = 0."""
    pp = tabs.pp
    rad = tabs.radnl
    r = 0.5 * (rad[1:] + rad[:-1])
    dr = rad[1:] - rad[:-1]
    vav = 0.5 * (tabs.vloctbl[1:] + tabs.vloctbl[:-1])
    g = np.asarray(g, dtype=np.float64)
    out = np.zeros(g.size)
    zero = g == 0.0
    out[zero] = np.sum(4 * np.pi * (r ** 2 * vav + r * pp.zps) * dr)
    gg = g[~zero][:, None]
    out[~zero] = np.sum(4 * np.pi * np.sin(gg * r[None, :]) / gg * (r[None, :] * vav[None, :] + pp.zps) * dr[None, :],
                        axis=1)
    return out


def calc_vpsl(tabs: PPTables, NLx, NLy, NLz, aL, Rion):
    """Vpsl(r) = Re sum_G Vion(G) exp(iG.r) with Vion(G) = sum_a [dVloc(G) -
    4pi Zps/G^2 (G != 0)] exp(-iG.R_a) / |cell| (prep_pp.f90:88-133).  The sum
    over the G set is an inverse DFT on the grid, taken by FFT.
    Returns (Vpsl (NL,), dVloc(G) (NL,), G vectors)."""
    aL = np.asarray(aL, dtype=np.float64)
    gx, gy, gz, m0 = g_vectors(NLx, NLy, NLz, aL)
    g2 = gx * gx + gy * gy + gz * gz
    dvloc = calc_vloc(tabs, np.sqrt(g2))
    alxyz = float(aL[0] * aL[1] * aL[2])
    coul = np.zeros_like(g2)
    nz = np.arange(g2.size) != m0
    coul[nz] = 4 * np.pi / g2[nz] * tabs.pp.zps
    vion = np.zeros(g2.size, np.complex128)
    for R in np.asarray(Rion, dtype=np.float64):
        vion += (dvloc - coul) * np.exp(-1j * (gx * R[0] + gy * R[1] + gz * R[2])) / alxyz
    # G index m in [-N/2, N/2) maps to the DFT bin m mod N
    grid = np.zeros((NLx, NLy, NLz), np.complex128)
    mx = np.arange(-(NLx // 2), NLx - NLx // 2) % NLx
    my = np.arange(-(NLy // 2), NLy - NLy // 2) % NLy
    mz = np.arange(-(NLz // 2), NLz - NLz // 2) % NLz
    grid[np.ix_(mx, my, mz)] = vion.reshape(NLx, NLy, NLz)
    vpsl = np.real(np.fft.ifftn(grid)) * (NLx * NLy * NLz)
    return np.ascontiguousarray(vpsl.ravel()), dvloc, (gx, gy, gz, m0)


def from_npz(path: str, lloc: int, lmax_ps: int = -1) -> RadialPP:
    """A RadialPP from tables saved in file units (the layout that
    tests/golden/make_testsuite_golden.py writes for a KY file)."""
    d = np.load(path)
    return from_tables(int(d["mr"]), float(d["step"]), int(d["mlps"]), float(d["zps"]), d["rrc"], d["vpp"],
                       d["upp"], lloc, lmax_ps)


def ewald_energy(Rion, zps, aL, grid, n_ewald: int = 4, a_ewald: float = 0.5):
    """Ion-ion energy by the Ewald sum of Total_Energy_omp (common/total_energy.f90:
    58-108) with the defaults newald = 4, aewald = 0.5 (io/inputoutput.f90:786-787):
    real-space images |n| <= n_ewald, the reciprocal sum over the grid's G set
    (G != 0) with rho_ion(G) = sum_a Z_a e^{-iG.R_a} / |cell|, and the
    self and neutralising-background terms.  zps: charge per atom."""
    from math import erfc, pi, sqrt
    Rion = np.asarray(Rion, dtype=np.float64)
    z = np.broadcast_to(np.asarray(zps, dtype=np.float64), (Rion.shape[0],))
    aL = np.asarray(aL, dtype=np.float64)
    alxyz = float(aL[0] * aL[1] * aL[2])
    e_real = 0.0
    rng_ = range(-n_ewald, n_ewald + 1)
    for ia in range(Rion.shape[0]):
        for ix in rng_:
            for iy in rng_:
                for iz in rng_:
                    shift = np.array([ix, iy, iz]) * aL
                    for ib in range(Rion.shape[0]):
                        if ix == 0 and iy == 0 and iz == 0 and ia == ib:
                            continue
                        rab = Rion[ia] - shift - Rion[ib]
                        r = sqrt(float(rab @ rab))
                        e_real += 0.5 * z[ia] * z[ib] * erfc(sqrt(a_ewald) * r) / r
    gx, gy, gz, m0 = g_vectors(*grid, aL)
    g2 = gx * gx + gy * gy + gz * gz
    rho = np.zeros(g2.size, np.complex128)
    for a in range(Rion.shape[0]):
        rho += z[a] * np.exp(-1j * (gx * Rion[a, 0] + gy * Rion[a, 1] + gz * Rion[a, 2])) / alxyz
    nz = np.arange(g2.size) != m0
    e_g = float(np.sum(alxyz * (4 * pi / g2[nz]) * np.abs(rho[nz]) ** 2 * np.exp(-g2[nz] / (4 * a_ewald)) * 0.5))
    e_self = -pi * float(z.sum()) ** 2 / (2 * a_ewald * alxyz) - sqrt(a_ewald / pi) * float((z * z).sum())
    return e_real + e_g + e_self
