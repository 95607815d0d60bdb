"""Host-side description of one periodic (ARTED) system.

Mirrors the module data SALMON builds before its real-time loop, with the same
names and the same Fortran (column-major) layouts, so that arrays move between
this package, the C ABI and a Fortran caller unchanged.  numpy arrays are kept
in C order with the Fortran axes reversed, e.g. ``zu(NL,NBoccmax,NK_s:NK_e)`` is
a C-order array of shape ``(nk_local, NBoccmax, NL)``.

Reference routines restated here (paths relative to the SALMON source tree):
  fd_coef            preparation/fd_coef.f90:20-83
  uniform k grid     preparation/init.f90:283-300 (Sym=1)
  occupations        preparation/init.f90:91-95
  sphere points      atom/pp/prep_pp.f90:263-347 (calc_jxyz, iperiodic=3)
  Jxyz linear index  preparation/prep_ps.f90:120
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

ND = 4  # global_variables.f90:41

# Reduced coordinates of the 8-atom diamond Si cell used by SALMON's bulk Si
# tests (testsuites/002_bulk_rt/inputfile, &atomic_red_coor).
DIAMOND_RED = np.array(
    [[0.00, 0.00, 0.00], [0.25, 0.25, 0.25], [0.50, 0.00, 0.50], [0.00, 0.50, 0.50],
     [0.50, 0.50, 0.00], [0.75, 0.25, 0.75], [0.25, 0.75, 0.75], [0.75, 0.75, 0.25]])


def fd_coef(nd: int = ND):
    """Central-difference coefficients lap(-nd:nd), nab(-nd:nd) before scaling.

    Same closed-form products as preparation/fd_coef.f90:26-73.
    Returns two arrays indexed n + nd.
    """
    n = nd
    lap = np.zeros(2 * n + 1)
    nab = np.zeros(2 * n + 1)
    s = 0.0
    for i in range(-n, n + 1):
        if i == 0:
            continue
        for j in range(-n, n + 1):
            if j == i or j == 0:
                continue
            s += 1.0 / (i * j)
    lap[n] = s
    for j in range(1, n + 1):
        t = 1.0
        for i in range(-n, n + 1):
            if i != j:
                t *= (j - i)
        s = 0.0
        for k in range(-n, n + 1):
            if k == j or k == 0:
                continue
            s0 = 1.0
            for i in range(-n, n + 1):
                if i in (k, j, 0):
                    continue
                s0 *= -i
            s += s0
        lap[n + j] = 2.0 * s / t
        lap[n - j] = lap[n + j]
    for j in range(1, n + 1):
        t = 1.0
        for i in range(-n, n + 1):
            if i != j:
                t *= (j - i)
        s = 1.0
        for i in range(-n, n + 1):
            if i in (j, 0):
                continue
            s *= -i
        nab[n + j] = s / t
        nab[n - j] = -nab[n + j]
    return lap, nab


def uniform_k_grid(nkx: int, nky: int, nkz: int, bl):
    """kAc(NK,3) of init_uniform_k_grid with Sym=1 (init.f90:288-300).

    Returned C-order with shape (3, NK) (Fortran kAc(NK,3))."""
    ks = []
    for ix in range(1, nkx + 1):
        for iy in range(1, nky + 1):
            for iz in range(1, nkz + 1):
                ks.append([-bl[0] / 2 + (ix - 0.5) * bl[0] / nkx,
                           -bl[1] / 2 + (iy - 0.5) * bl[1] / nky,
                           -bl[2] / 2 + (iz - 0.5) * bl[2] / nkz])
    return np.ascontiguousarray(np.array(ks).T)


class SgpuDesc(C.Structure):
    """ctypes mirror of ``sgpu_desc`` (include/salmon_gpu.h)."""
    _fields_ = [
        ("NLx", C.c_int32), ("NLy", C.c_int32), ("NLz", C.c_int32),
        ("Hx", C.c_double), ("Hy", C.c_double), ("Hz", C.c_double),
        ("aLx", C.c_double), ("aLy", C.c_double), ("aLz", C.c_double),
        ("NK", C.c_int32), ("NK_s", C.c_int32), ("NK_e", C.c_int32),
        ("NB", C.c_int32), ("NBoccmax", C.c_int32),
        ("lapx", C.c_double * 5), ("lapy", C.c_double * 5), ("lapz", C.c_double * 5),
        ("nabx", C.c_double * 5), ("naby", C.c_double * 5), ("nabz", C.c_double * 5),
        ("NI", C.c_int32), ("Nps", C.c_int32), ("Nlma", C.c_int32),
        ("Mps", C.POINTER(C.c_int32)), ("Jxyz", C.POINTER(C.c_int32)),
        ("Jxx", C.POINTER(C.c_int32)), ("Jyy", C.POINTER(C.c_int32)), ("Jzz", C.POINTER(C.c_int32)),
        ("uV", C.POINTER(C.c_double)), ("iuV", C.POINTER(C.c_int32)),
        ("a_tbl", C.POINTER(C.c_int32)), ("occ", C.POINTER(C.c_double)),
    ]


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class System:
    """Grid, k-points, occupations and Kleinman-Bylander tables of one system."""
    NLx: int
    NLy: int
    NLz: int
    aL: np.ndarray                      # (3,) cell lengths
    kAc0: np.ndarray                    # (3, NK)  kAc0(NK,3)
    NB: int
    NBoccmax: int
    occ: np.ndarray                     # (NK, NB) occ(NB,NK)
    Rion: np.ndarray                    # (NI, 3)  Rion(3,NI)
    Rps: float                          # projector sphere radius
    Mps: np.ndarray                     # (NI,)
    Jxyz: np.ndarray                    # (NI, Nps) 1-based
    Jxx: np.ndarray
    Jyy: np.ndarray
    Jzz: np.ndarray
    uV: np.ndarray                      # (Nlma, Nps)
    iuV: np.ndarray                     # (Nlma,)
    a_tbl: np.ndarray                   # (Nlma,) 1-based
    NK_s: int = 1
    NK_e: int = 0
    extra: dict = field(default_factory=dict)

    def __post_init__(self):
        if self.NK_e == 0:
            self.NK_e = self.NK

    # ---- derived quantities (global_variables.f90) ----
    @property
    def NL(self):
        return self.NLx * self.NLy * self.NLz

    @property
    def NK(self):
        return self.kAc0.shape[1]

    @property
    def nk_local(self):
        return self.NK_e - self.NK_s + 1

    @property
    def H(self):
        return self.aL / np.array([self.NLx, self.NLy, self.NLz])

    @property
    def Hxyz(self):
        h = self.H
        return float(h[0] * h[1] * h[2])

    @property
    def aLxyz(self):
        return float(self.aL[0] * self.aL[1] * self.aL[2])

    @property
    def NI(self):
        return self.Mps.shape[0]

    @property
    def Nps(self):
        return self.Jxyz.shape[1]

    @property
    def Nlma(self):
        return self.uV.shape[0]

    def lap_nab(self):
        """lapx..nabz(0:4) scaled by 1/H^2 and 1/H (fd_coef.f90:75-80)."""
        lap, nab = fd_coef()
        h = self.H
        out = {}
        for d, ax in enumerate("xyz"):
            out["lap" + ax] = lap[ND:] / h[d] ** 2
            out["nab" + ax] = nab[ND:] / h[d]
        return out

    def grid_coords(self):
        """Lx, Ly, Lz of every grid point (init.f90:20-30), 0-based index order."""
        ix, iy, iz = np.meshgrid(np.arange(self.NLx), np.arange(self.NLy), np.arange(self.NLz), indexing="ij")
        return ix.ravel(), iy.ravel(), iz.ravel()

    def desc(self) -> SgpuDesc:
        """Builds the C descriptor; the arrays it points to are owned by self."""
        for name in ("Mps", "Jxyz", "Jxx", "Jyy", "Jzz", "iuV", "a_tbl"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.int32))
        for name in ("uV", "occ"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.float64))
        d = SgpuDesc()
        d.NLx, d.NLy, d.NLz = self.NLx, self.NLy, self.NLz
        d.Hx, d.Hy, d.Hz = (float(v) for v in self.H)
        d.aLx, d.aLy, d.aLz = (float(v) for v in self.aL)
        d.NK, d.NK_s, d.NK_e = self.NK, self.NK_s, self.NK_e
        d.NB, d.NBoccmax = self.NB, self.NBoccmax
        ln = self.lap_nab()
        for key in ("lapx", "lapy", "lapz", "nabx", "naby", "nabz"):
            arr = getattr(d, key)
            for n in range(5):
                arr[n] = float(ln[key][n])
        d.NI, d.Nps, d.Nlma = self.NI, self.Nps, self.Nlma
        d.Mps, d.Jxyz, d.Jxx, d.Jyy, d.Jzz = (_ip(self.Mps), _ip(self.Jxyz), _ip(self.Jxx), _ip(self.Jyy),
                                              _ip(self.Jzz))
        d.uV, d.iuV, d.a_tbl, d.occ = _dp(self.uV), _ip(self.iuV), _ip(self.a_tbl), _dp(self.occ)
        self._desc_keepalive = d
        return d

    def sphere_positions(self):
        """x,y,z of point j of atom a relative to the cell image, as used by
        update_projector and current (projector.f90:61, current.f90:253-255).
        Shape (NI, Nps, 3)."""
        h = self.H
        i = self.Jxyz - 1
        lx = i // (self.NLy * self.NLz)
        ly = (i // self.NLz) % self.NLy
        lz = i % self.NLz
        return np.stack([lx * h[0] - self.Jxx * self.aL[0],
                         ly * h[1] - self.Jyy * self.aL[1],
                         lz * h[2] - self.Jzz * self.aL[2]], axis=-1)


def calc_jxyz(NLx, NLy, NLz, aL, Rion, Rps):
    """Sphere points of every atom, in the order of calc_jxyz with nc=2
    (atom/pp/prep_pp.f90:314-345): images ix,iy,iz in -2..2, then grid points in
    index order.  Returns Mps (NI,), Jxyz (1-based), Jxx, Jyy, Jzz as (NI, Nps)
    and the distance components (NI, Nps, 3) from the atom image."""
    h = np.asarray(aL) / np.array([NLx, NLy, NLz])
    N = (NLx, NLy, NLz)
    per_atom = []
    for a in range(Rion.shape[0]):
        js, jx, jy, jz, dv = [], [], [], [], []
        for ax in range(-2, 3):
            for ay in range(-2, 3):
                for az in range(-2, 3):
                    t = Rion[a] + np.array([ax, ay, az]) * np.asarray(aL)
                    # only the grid box around the image can be inside the sphere; the box
                    # is enumerated in grid-index order, like the full grid
                    lo = [max(0, int(np.floor((t[d] - Rps) / h[d]))) for d in range(3)]
                    hi = [min(N[d] - 1, int(np.ceil((t[d] + Rps) / h[d]))) for d in range(3)]
                    if any(lo[d] > hi[d] for d in range(3)):
                        continue
                    bx, by, bz = np.meshgrid(np.arange(lo[0], hi[0] + 1), np.arange(lo[1], hi[1] + 1),
                                             np.arange(lo[2], hi[2] + 1), indexing="ij")
                    mx, my, mz = bx.ravel(), by.ravel(), bz.ravel()
                    x = mx * h[0] - t[0]
                    y = my * h[1] - t[1]
                    z = mz * h[2] - t[2]
                    r = np.sqrt(x * x + y * y + z * z)
                    sel = np.nonzero(r < Rps)[0]
                    if sel.size:
                        js.append(mz[sel] + 1 + NLz * my[sel] + NLy * NLz * mx[sel])
                        jx.append(np.full(sel.size, ax)); jy.append(np.full(sel.size, ay))
                        jz.append(np.full(sel.size, az))
                        dv.append(np.stack([x[sel], y[sel], z[sel]], axis=1))
        per_atom.append((np.concatenate(js), np.concatenate(jx), np.concatenate(jy), np.concatenate(jz),
                         np.concatenate(dv)))
    NI = Rion.shape[0]
    Mps = np.array([p[0].size for p in per_atom], dtype=np.int32)
    Nps = int(Mps.max())
    Jxyz = np.zeros((NI, Nps), np.int32)
    Jxx = np.zeros((NI, Nps), np.int32)
    Jyy = np.zeros((NI, Nps), np.int32)
    Jzz = np.zeros((NI, Nps), np.int32)
    dist = np.zeros((NI, Nps, 3))
    for a, (js, jx, jy, jz, dv) in enumerate(per_atom):
        m = js.size
        Jxyz[a, :m], Jxx[a, :m], Jyy[a, :m], Jzz[a, :m], dist[a, :m] = js, jx, jy, jz, dv
    return Mps, Jxyz, Jxx, Jyy, Jzz, dist


def gaussian_projectors(Mps, dist, Hxyz, rc=2.0):
    """s + (px,py,pz) projectors per atom: radial exp(-r^2/rc^2) times 1, x, y, z,
    each normalised so that sum_j uV^2 Hxyz = 1; iuV = +1 (s), -1 (p).  Projectors
    are numbered atom by atom, as set_lma_tbl does."""
    NI, Nps = dist.shape[:2]
    uV = np.zeros((NI * 4, Nps))
    iuV = np.zeros(NI * 4, np.int32)
    a_tbl = np.zeros(NI * 4, np.int32)
    for a in range(NI):
        m = Mps[a]
        d = dist[a, :m]
        r2 = (d * d).sum(axis=1)
        rad = np.exp(-r2 / rc ** 2)
        for p, ang in enumerate([np.ones(m), d[:, 0], d[:, 1], d[:, 2]]):
            v = rad * ang
            v = v / np.sqrt((v * v).sum() * Hxyz)
            uV[4 * a + p, :m] = v
            iuV[4 * a + p] = 1 if p == 0 else -1
            a_tbl[4 * a + p] = a + 1
    return uV, iuV, a_tbl


def periodic_gaussian_vloc(NLx, NLy, NLz, aL, centres, depth, width, cutoff=None):
    """V(r) = -sum_a D_a exp(-|r-R_a|^2/w_a^2) summed over the 27 nearest images.
    With `cutoff` (in widths), an image only adds to the grid box within
    cutoff*w of it (a large cell's potential in seconds instead of minutes; the
    dropped terms are below exp(-cutoff^2) of the depth)."""
    h = np.asarray(aL) / np.array([NLx, NLy, NLz])
    N = (NLx, NLy, NLz)
    if cutoff is None:
        ix, iy, iz = np.meshgrid(np.arange(NLx), np.arange(NLy), np.arange(NLz), indexing="ij")
        r = np.stack([ix.ravel() * h[0], iy.ravel() * h[1], iz.ravel() * h[2]], axis=1)
        v = np.zeros(r.shape[0])
        for a in range(centres.shape[0]):
            for ax in (-1, 0, 1):
                for ay in (-1, 0, 1):
                    for az in (-1, 0, 1):
                        c = centres[a] + np.array([ax, ay, az]) * aL
                        d2 = ((r - c) ** 2).sum(axis=1)
                        v -= depth[a] * np.exp(-d2 / width[a] ** 2)
        return v
    v = np.zeros((NLx, NLy, NLz))
    for a in range(centres.shape[0]):
        rc = cutoff * width[a]
        for ax in (-1, 0, 1):
            for ay in (-1, 0, 1):
                for az in (-1, 0, 1):
                    c = centres[a] + np.array([ax, ay, az]) * aL
                    lo = [max(0, int(np.floor((c[d] - rc) / h[d]))) for d in range(3)]
                    hi = [min(N[d] - 1, int(np.ceil((c[d] + rc) / h[d]))) for d in range(3)]
                    if any(lo[d] > hi[d] for d in range(3)):
                        continue
                    gx = np.arange(lo[0], hi[0] + 1) * h[0] - c[0]
                    gy = np.arange(lo[1], hi[1] + 1) * h[1] - c[1]
                    gz = np.arange(lo[2], hi[2] + 1) * h[2] - c[2]
                    d2 = gx[:, None, None] ** 2 + gy[None, :, None] ** 2 + gz[None, None, :] ** 2
                    v[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1] -= depth[a] * np.exp(-d2 / width[a] ** 2)
    return v.ravel()


def orthonormalise(zu, Hxyz):
    """Orthonormalises the bands of every k-point under <a|b> = Hxyz sum conj(a) b
    (Householder QR; the span equals that of Gram-Schmidt).  zu: (nk, nb, NL)."""
    out = np.empty_like(zu)
    for k in range(zu.shape[0]):
        q, r = np.linalg.qr(zu[k].T)
        ph = np.sign(np.real(np.diag(r)))
        ph[ph == 0] = 1
        out[k] = (q * ph).T / np.sqrt(Hxyz)
    return out


SEED = 20261203


def microbench_system(N: int, nkgrid=(4, 4, 4), Nb: int = 32, A=(1e-2, 0.0, 0.0), a: float = 10.26,
                      seed: int = SEED, with_orbitals: bool = True, nk_limit: int | None = None):
    """The hpsi/Taylor operator microbench system: cubic cell a=10.26 bohr, grid
    N^3, uniform k grid shifted by A, Nb bands, V_loc = 8 seeded periodic
    Gaussians (depth U(0.5,2) Ha, width U(1,2) bohr) on the diamond sites,
    8 atoms x {s,px,py,pz} Gaussian projectors (r_c = 2 bohr, R_ps = 2 bohr).

    Returns (system, kAc (3,NK), Vloc (NL,), zu (nk,Nb,NL) complex128 or None).
    ``nk_limit`` keeps only the first k-points (small test cases)."""
    rng = np.random.default_rng(seed)
    aL = np.array([a, a, a])
    bl = 2 * np.pi / aL
    kAc0 = uniform_k_grid(*nkgrid, bl)
    if nk_limit is not None:
        kAc0 = np.ascontiguousarray(kAc0[:, :nk_limit])
    NK = kAc0.shape[1]
    nkxyz = nkgrid[0] * nkgrid[1] * nkgrid[2]
    occ = np.full((NK, Nb), 2.0 / nkxyz)
    Rion = DIAMOND_RED * aL
    Mps, Jxyz, Jxx, Jyy, Jzz, dist = calc_jxyz(N, N, N, aL, Rion, 2.0)
    Hxyz = float(np.prod(aL / N))
    uV, iuV, a_tbl = gaussian_projectors(Mps, dist, Hxyz)
    depth = rng.uniform(0.5, 2.0, Rion.shape[0])
    width = rng.uniform(1.0, 2.0, Rion.shape[0])
    vloc = periodic_gaussian_vloc(N, N, N, aL, Rion, depth, width)
    sysm = System(NLx=N, NLy=N, NLz=N, aL=aL, kAc0=kAc0, NB=Nb, NBoccmax=Nb, occ=occ, Rion=Rion, Rps=2.0,
                  Mps=Mps, Jxyz=Jxyz, Jxx=Jxx, Jyy=Jyy, Jzz=Jzz, uV=uV, iuV=iuV, a_tbl=a_tbl)
    sysm.extra.update(seed=seed, depth=depth, width=width)
    kAc = np.ascontiguousarray(kAc0 + np.asarray(A, dtype=np.float64)[:, None])
    zu = None
    if with_orbitals:
        NL = N ** 3
        zu = rng.standard_normal((NK, Nb, NL)) + 1j * rng.standard_normal((NK, Nb, NL))
        zu = orthonormalise(zu, Hxyz)
    return sysm, kAc, vloc, zu


def si_supercell_system(ncell=(1, 1, 1), grid=(16, 16, 16), nkgrid=(4, 4, 4), Nb: int = 16, A=(0.0, 0.0, 0.0),
                        a: float = 10.26, seed: int = SEED, with_orbitals: bool = True, Nocc: int | None = None):
    """Diamond-Si supercell of ncell cubic 8-atom cells (a = 10.26 bohr) on the
    given grid: 8*prod(ncell) atoms x {s,px,py,pz} Gaussian projectors (r_c =
    R_ps = 2 bohr), V_loc = seeded periodic Gaussians on the atoms, uniform
    nkgrid k-points, Nb bands of which the lowest Nocc (default all) are occupied
    (2/NK each) and propagated in real time.  The shapes of the Si8 / Si16 / Si64 systems:
    ncell (1,1,1) 16^3, (1,1,2) 16x16x32, (2,2,2) 32^3.
    Returns (system, kAc (3,NK), Vloc (NL,), zu (nk,Nb,NL) complex128 or None)."""
    rng = np.random.default_rng(seed)
    nc = np.asarray(ncell)
    aL = a * nc.astype(np.float64)
    NLx, NLy, NLz = grid
    bl = 2 * np.pi / aL
    kAc0 = uniform_k_grid(*nkgrid, bl)
    NK = kAc0.shape[1]
    Nocc = Nb if Nocc is None else Nocc
    occ = np.zeros((NK, Nb))
    occ[:, :Nocc] = 2.0 / NK
    cells = np.array([[i, j, k] for i in range(nc[0]) for j in range(nc[1]) for k in range(nc[2])])
    Rion = np.concatenate([(DIAMOND_RED + c) * a for c in cells])
    Mps, Jxyz, Jxx, Jyy, Jzz, dist = calc_jxyz(NLx, NLy, NLz, aL, Rion, 2.0)
    Hxyz = float(np.prod(aL / np.array(grid)))
    uV, iuV, a_tbl = gaussian_projectors(Mps, dist, Hxyz)
    depth = rng.uniform(0.5, 2.0, Rion.shape[0])
    width = rng.uniform(1.0, 2.0, Rion.shape[0])
    # large supercells: images only near the grid box they reach (see periodic_gaussian_vloc)
    vloc = periodic_gaussian_vloc(NLx, NLy, NLz, aL, Rion, depth, width, cutoff=8.0 if Rion.shape[0] > 64 else None)
    sysm = System(NLx=NLx, NLy=NLy, NLz=NLz, aL=aL, kAc0=kAc0, NB=Nb, NBoccmax=Nocc, occ=occ, Rion=Rion, Rps=2.0,
                  Mps=Mps, Jxyz=Jxyz, Jxx=Jxx, Jyy=Jyy, Jzz=Jzz, uV=uV, iuV=iuV, a_tbl=a_tbl)
    sysm.extra.update(seed=seed, depth=depth, width=width)
    kAc = np.ascontiguousarray(kAc0 + np.asarray(A, dtype=np.float64)[:, None])
    zu = None
    if with_orbitals:
        NL = NLx * NLy * NLz
        zu = rng.standard_normal((NK, Nb, NL)) + 1j * rng.standard_normal((NK, Nb, NL))
        zu = orthonormalise(zu, Hxyz)
    return sysm, kAc, vloc, zu


BATCHED_SYSTEMS = {  # name: (ncell, grid, nkgrid, bands)
    "Si8": ((1, 1, 1), (16, 16, 16), (4, 4, 4), 16),
    "Si16": ((1, 1, 2), (16, 16, 32), (4, 4, 2), 32),
    "Si64": ((2, 2, 2), (32, 32, 32), (2, 2, 2), 128),
}


def small_system(NLx=8, NLy=8, NLz=10, nk=3, nb=4, a=(6.0, 6.5, 7.0), nat=2, seed=7, Rps=1.6):
    """A small non-cubic system with ragged sizes for exhaustive parity tests:
    uneven grid, few k-points and bands, random atom sites, Gaussian projectors."""
    rng = np.random.default_rng(seed)
    aL = np.asarray(a, dtype=np.float64)
    kAc0 = np.ascontiguousarray(rng.uniform(-0.5, 0.5, (3, nk)))
    occ = rng.uniform(0.1, 1.0, (nk, nb))
    Rion = rng.uniform(0, 1, (nat, 3)) * aL
    Mps, Jxyz, Jxx, Jyy, Jzz, dist = calc_jxyz(NLx, NLy, NLz, aL, Rion, Rps)
    Hxyz = float(np.prod(aL / np.array([NLx, NLy, NLz])))
    uV, iuV, a_tbl = gaussian_projectors(Mps, dist, Hxyz, rc=Rps)
    vloc = periodic_gaussian_vloc(NLx, NLy, NLz, aL, Rion, rng.uniform(0.5, 2, nat), rng.uniform(1, 2, nat))
    sysm = System(NLx=NLx, NLy=NLy, NLz=NLz, aL=aL, kAc0=kAc0, NB=nb, NBoccmax=nb, occ=occ, Rion=Rion, Rps=Rps,
                  Mps=Mps, Jxyz=Jxyz, Jxx=Jxx, Jyy=Jyy, Jzz=Jzz, uV=uV, iuV=iuV, a_tbl=a_tbl)
    kAc = np.ascontiguousarray(kAc0 + rng.uniform(-0.05, 0.05, (3, 1)))
    NL = NLx * NLy * NLz
    zu = rng.standard_normal((nk, nb, NL)) + 1j * rng.standard_normal((nk, nb, NL))
    zu = orthonormalise(zu, Hxyz)
    return sysm, kAc, vloc, zu


def si_pp_system(tabs, ncell=(1, 1, 1), grid=(8, 8, 8), nkgrid=(4, 4, 4), NB: int = 32, Nocc: int = 16,
                 a: float = 10.26, seed: int = SEED, with_orbitals: bool = True, kpoints=None):
    """Diamond-Si supercell with the physical pseudopotential ``tabs``
    (``pseudo.prepare`` of a KY file): sphere points within the element's Rps
    (calc_jxyz), uV = spline(udV_l) x Ylm on them (calc_uv), Vpsl from the
    structure factor (calc_vpsl); NB bands of which the lowest Nocc carry
    occ = 2/NK (init.f90:91-95).  The shape of SALMON's bulk-Si testsuites
    (001_bulk_gs, 002_bulk_rt) is the default: 8 atoms, 8^3 grid, 4^3 k, 32 bands.
    Returns (system, kAc0 (3,NK), Vpsl (NL,), zu_GS (nk,NB,NL) or None); zu_GS
    is seeded random and orthonormal (the reference's init_wf draws random
    orbitals too).  kpoints (3, NK), if given, replaces the uniform k grid."""
    from . import pseudo as P
    nc = np.asarray(ncell)
    aL = a * nc.astype(np.float64)
    NLx, NLy, NLz = grid
    bl = 2 * np.pi / aL
    kAc0 = uniform_k_grid(*nkgrid, bl) if kpoints is None else np.ascontiguousarray(kpoints, dtype=np.float64)
    NK = kAc0.shape[1]
    occ = np.zeros((NK, NB))
    occ[:, :Nocc] = 2.0 / NK
    cells = np.array([[i, j, k] for i in range(nc[0]) for j in range(nc[1]) for k in range(nc[2])])
    Rion = np.concatenate([(DIAMOND_RED + c) * a for c in cells])
    rps = tabs.pp.rps
    Mps, Jxyz, Jxx, Jyy, Jzz, dist = calc_jxyz(NLx, NLy, NLz, aL, Rion, rps)
    uV, iuV, a_tbl = P.kb_tables(tabs, Mps, dist)
    vpsl, _, _ = P.calc_vpsl(tabs, NLx, NLy, NLz, aL, Rion)
    sysm = System(NLx=NLx, NLy=NLy, NLz=NLz, aL=aL, kAc0=kAc0, NB=NB, NBoccmax=Nocc, occ=occ, Rion=Rion, Rps=rps,
                  Mps=Mps, Jxyz=Jxyz, Jxx=Jxx, Jyy=Jyy, Jzz=Jzz, uV=uV, iuV=iuV, a_tbl=a_tbl)
    sysm.extra.update(seed=seed, zps=tabs.pp.zps)
    zu = None
    if with_orbitals:
        rng = np.random.default_rng(seed)
        NL = NLx * NLy * NLz
        zu = rng.standard_normal((NK, NB, NL)) + 1j * rng.standard_normal((NK, NB, NL))
        zu = orthonormalise(zu, sysm.Hxyz)
    return sysm, np.ascontiguousarray(kAc0), vpsl, zu


def folded_kpoints(ks_super, ncell, aL_super):
    """The unit-cell k-points that fold onto the supercell k-points ks_super
    (3, NKs) of a supercell of ncell unit cells: k_u = k_s + m b_s for every
    m in [0, ncell), b_s = 2 pi / aL_super per axis.  Returns (3, NKs * prod(ncell))
    ordered supercell k-point by supercell k-point, m in C order."""
    nc = np.asarray(ncell)
    bs = 2 * np.pi / np.asarray(aL_super, dtype=np.float64)
    ms = np.array([[i, j, k] for i in range(nc[0]) for j in range(nc[1]) for k in range(nc[2])], dtype=np.float64)
    out = [ks_super[:, s] + m * bs for s in range(ks_super.shape[1]) for m in ms]
    return np.ascontiguousarray(np.array(out).T), ms.astype(np.int64)


def unfold_to_supercell(zu_cell, ncell, ms, nks, grid_cell):
    """Bloch-periodic parts on the supercell grid from those of the unit cell
    (torch CUDA tensors): for supercell k-point s and unit-cell k-point
    k_u = k_s + m b_s, u_s(R) = exp(i m b_s . R h) u_{k_u}(R mod cell) / sqrt(prod
    ncell), an eigenstate of the supercell Hamiltonian at k_s with the same
    eigenvalue (a perfect crystal).  zu_cell: (nks * nfold, nb, NLc) complex128;
    returns (nks, nfold * nb, NLs) with the unit-cell k-points of one supercell
    k-point band-block after band-block."""
    import torch
    nc = [int(x) for x in ncell]
    gx, gy, gz = grid_cell
    Sx, Sy, Sz = gx * nc[0], gy * nc[1], gz * nc[2]
    nfold = int(np.prod(nc))
    nb = zu_cell.shape[1]
    out = torch.empty((nks, nfold * nb, Sx * Sy * Sz), dtype=torch.complex128, device=zu_cell.device)
    ax = [torch.arange(n, device=zu_cell.device, dtype=torch.float64) for n in (Sx, Sy, Sz)]
    for s in range(nks):
        for j in range(nfold):
            m = ms[j]
            u = zu_cell[s * nfold + j].reshape(nb, gx, gy, gz).repeat(1, nc[0], nc[1], nc[2])
            ph = [torch.exp(1j * 2 * np.pi * float(m[d]) * ax[d] / (nc[d] * (gx, gy, gz)[d])) for d in range(3)]
            phase = ph[0][:, None, None] * ph[1][None, :, None] * ph[2][None, None, :]
            out[s, j * nb:(j + 1) * nb] = (u * phase[None] / np.sqrt(nfold)).reshape(nb, -1)
    return out
