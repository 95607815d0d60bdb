"""ctypes front end of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

``liboracle.so``            C restatement of SALMON's RT hot path (salmon_oracle.c)
``_ref/libsalmon_ref.so``   SALMON's own AVX stencils compiled from the reference
                            tree, plus a Taylor-step driver (ref_driver.c)

Only tests/, the smoke check and bench.py's CPU-baseline legs import this
module.  Arrays follow salmon_b200.system conventions (C order, Fortran axes
reversed).  Every function returns new arrays; inputs are not modified unless
stated.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


# Where the SALMON source tree is read from: the REF_ROOT environment variable,
# else this recipe's one default location (the same default as oracle/Makefile).
# Only the recipes (this build, the Makefile, tests/golden/*.py) read the tree;
# machines without it use the prebuilt _ref library and the committed fixtures.
_REF_ROOT_DEFAULT = "/root/reference"


def ref_root():
    """The SALMON source tree, or None when it is not present on this machine."""
    root = os.environ.get("REF_ROOT") or _REF_ROOT_DEFAULT
    return root if os.path.isdir(os.path.join(root, "src", "ARTED")) else None


def build(quiet=True):
    """Builds liboracle.so, and _ref/libsalmon_ref.so when the reference tree
    is present (oracle/Makefile)."""
    targets = ["liboracle.so"]
    env = dict(os.environ)
    root = ref_root()
    if root and os.path.isdir(os.path.join(root, "src", "ARTED", "stencil", "C", "AVX")):
        targets.append("ref")
        env["REF_ROOT"] = root
    out = subprocess.run(["make", "-C", HERE] + targets, capture_output=True, text=True, env=env)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        L = _LIB
        for name in ("orc_fd_coef", "orc_stencil", "orc_update_projector", "orc_hpsi", "orc_hamiltonian",
                     "orc_psi_rho", "orc_current", "orc_energy_terms", "orc_gram_schmidt", "orc_cg",
                     "orc_subspace_h"):
            getattr(L, name).restype = None
        L.orc_max_threads.restype = C.c_int
    return _LIB


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libsalmon_ref.so"))


def ref_lib():
    """The reference's compiled AVX stencils (raises if not built)."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libsalmon_ref.so")
        if not os.path.exists(path):
            build()
        _REF = C.CDLL(path)
        _REF.ref_set_grid.restype = C.c_int
        _REF.ref_hamiltonian.restype = C.c_int
        _REF.ref_max_threads.restype = C.c_int
        _REF.ref_stencil.restype = None
        _REF.ref_current_stencil.restype = None
        _REF.ref_total_energy_stencil.restype = None
    return _REF


def _aligned_complex(shape):
    """complex128 array with a 64-byte aligned base (the AVX kernels use aligned loads)."""
    n = int(np.prod(shape))
    raw = np.empty(n * 16 + 64, dtype=np.uint8)
    off = (-raw.ctypes.data) % 64
    return raw[off:off + n * 16].view(np.complex128).reshape(shape)


# ---------------------------------------------------------------- restatement
def fd_coef(nd=4):
    lap = np.zeros(2 * nd + 1)
    nab = np.zeros(2 * nd + 1)
    lib().orc_fd_coef(C.c_int(nd), _ptr(lap), _ptr(nab))
    return lap, nab


def stencil(sysm, A, B, Cc, D, E):
    """hpsi1_RT_stencil on one orbital (stencil/F90/hpsi.f90:27-198)."""
    d = sysm.desc()
    E = np.ascontiguousarray(E, dtype=np.complex128)
    F = np.empty_like(E)
    lib().orc_stencil(C.byref(d), C.c_double(A), _ptr(np.ascontiguousarray(B, np.float64)),
                      _ptr(np.ascontiguousarray(Cc, np.float64)), _ptr(np.ascontiguousarray(D, np.float64)),
                      _ptr(E), _ptr(F))
    return F


def update_projector(sysm, kAc):
    """(ekr (nkl,NI,Nps), zproj (nkl,Nlma,Nps)) of update_projector_omp."""
    d = sysm.desc()
    ekr = np.zeros((sysm.nk_local, sysm.NI, sysm.Nps), np.complex128)
    zproj = np.zeros((sysm.nk_local, sysm.Nlma, sysm.Nps), np.complex128)
    lib().orc_update_projector(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(ekr), _ptr(zproj))
    return ekr, zproj


def hpsi(sysm, kAc, vloc, zproj, ik, tpsi, want_tt=False):
    """hpsi_omp_KB_GS/RT for one orbital of k-point ik (1-based)."""
    d = sysm.desc()
    tpsi = np.ascontiguousarray(tpsi, dtype=np.complex128)
    h = np.empty_like(tpsi)
    tt = np.empty_like(tpsi) if want_tt else None
    lib().orc_hpsi(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(np.ascontiguousarray(vloc)),
                   _ptr(zproj), C.c_int(ik), _ptr(tpsi), _ptr(h), _ptr(tt) if want_tt else None)
    return (h, tt) if want_tt else h


def hamiltonian(sysm, kAc, vloc, zproj, dt, zu, nthreads=0):
    """One Taylor step (RT/hamiltonian.f90:27-123); returns the new zu."""
    d = sysm.desc()
    z = np.array(zu, dtype=np.complex128, order="C", copy=True)
    lib().orc_hamiltonian(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(np.ascontiguousarray(vloc)),
                          _ptr(zproj), C.c_double(dt), _ptr(z), C.c_int(nthreads))
    return z


def psi_rho(sysm, zu):
    d = sysm.desc()
    zu = np.ascontiguousarray(zu, dtype=np.complex128)
    rho = np.zeros(sysm.NL)
    lib().orc_psi_rho(C.byref(d), _ptr(zu), C.c_int(zu.shape[1]), _ptr(rho))
    return rho


def current(sysm, kAc, zu):
    """jav(3) before the allreduce; builds zproj for kAc like current() does."""
    d = sysm.desc()
    _, zproj = update_projector(sysm, kAc)
    zu = np.ascontiguousarray(zu, dtype=np.complex128)
    jav = np.zeros(3)
    lib().orc_current(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(zproj), _ptr(zu),
                      C.c_int(zu.shape[1]), _ptr(jav))
    return jav


def energy_terms(sysm, kAc, zu):
    d = sysm.desc()
    zu = np.ascontiguousarray(zu, dtype=np.complex128)
    ek, en = C.c_double(), C.c_double()
    lib().orc_energy_terms(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(zu), C.c_int(zu.shape[1]),
                           C.byref(ek), C.byref(en))
    return ek.value, en.value


def gram_schmidt(sysm, zu):
    d = sysm.desc()
    z = np.array(zu, dtype=np.complex128, order="C", copy=True)
    lib().orc_gram_schmidt(C.byref(d), _ptr(z))
    return z


def cg(sysm, kAc, vloc, zu, ncg):
    """CG_ompk; returns (zu, esp_var (nkl,NB), iterations (nkl,NB))."""
    d = sysm.desc()
    _, zproj = update_projector(sysm, kAc)
    z = np.array(zu, dtype=np.complex128, order="C", copy=True)
    esp = np.zeros((sysm.nk_local, sysm.NB))
    its = np.zeros((sysm.nk_local, sysm.NB), np.int32)
    lib().orc_cg(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(np.ascontiguousarray(vloc)),
                 _ptr(zproj), _ptr(z), C.c_int(ncg), _ptr(esp), _ptr(its, _ip))
    return z, esp, its


def subspace_h(sysm, kAc, vloc, zu, ik):
    """za(NB,NB) of diag_omp for k-point ik (1-based), returned as a numpy
    matrix M with M[row, col] = za(row+1, col+1)."""
    d = sysm.desc()
    _, zproj = update_projector(sysm, kAc)
    za = np.zeros((sysm.NB, sysm.NB), np.complex128)  # C-order [col][row] == Fortran (row,col)
    lib().orc_subspace_h(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(np.ascontiguousarray(vloc)),
                         _ptr(zproj), _ptr(np.ascontiguousarray(zu, dtype=np.complex128)), C.c_int(ik), _ptr(za))
    return za.T.copy()


def diag(sysm, kAc, vloc, zu):
    """diag_omp (GS/diag.f90:22-173): subspace H per k, eigh (zheev stand-in:
    scipy/numpy LAPACK), rotation zutmp(:,ib1) = sum_ib2 zu(:,ib2) za(ib2,ib1).
    Returns (zu, esp (nkl,NB))."""
    out = np.empty_like(zu)
    esp = np.zeros((sysm.nk_local, sysm.NB))
    for ikl in range(sysm.nk_local):
        M = subspace_h(sysm, kAc, vloc, zu, sysm.NK_s + ikl)
        w, V = np.linalg.eigh(M, UPLO="L")
        out[ikl] = V.T @ zu[ikl]
        esp[ikl] = w
    return out, esp


def max_threads():
    return lib().orc_max_threads()


# ----------------------------------------------------- the reference's own AVX
def ref_stencil(sysm, A, B, Cc, D, E):
    """SALMON's AVX hpsi1_rt_stencil_ (stencil/C/AVX/hpsi.c:35-148)."""
    R = ref_lib()
    if R.ref_set_grid(sysm.NLx, sysm.NLy, sysm.NLz) != 0:
        raise ValueError("the reference AVX stencil needs an even NLz")
    Ea = _aligned_complex(E.shape)
    Ea[...] = E
    F = _aligned_complex(E.shape)
    R.ref_stencil(C.c_double(A), _ptr(np.ascontiguousarray(B, np.float64)), _ptr(np.ascontiguousarray(Cc, np.float64)),
                  _ptr(np.ascontiguousarray(D, np.float64)), _ptr(Ea), _ptr(F))
    return np.array(F)


def ref_current_stencil(sysm, Cc, E):
    R = ref_lib()
    if R.ref_set_grid(sysm.NLx, sysm.NLy, sysm.NLz) != 0:
        raise ValueError("the reference AVX stencil needs an even NLz")
    Ea = _aligned_complex(E.shape)
    Ea[...] = E
    f, g, h = C.c_double(), C.c_double(), C.c_double()
    R.ref_current_stencil(_ptr(np.ascontiguousarray(Cc, np.float64)), _ptr(Ea), C.byref(f), C.byref(g), C.byref(h))
    return np.array([f.value, g.value, h.value])


def ref_total_energy_stencil(sysm, A, Cc, D, E):
    R = ref_lib()
    if R.ref_set_grid(sysm.NLx, sysm.NLy, sysm.NLz) != 0:
        raise ValueError("the reference AVX stencil needs an even NLz")
    Ea = _aligned_complex(E.shape)
    Ea[...] = E
    F = np.zeros(1, np.complex128)
    R.ref_total_energy_stencil(C.c_double(A), _ptr(np.ascontiguousarray(Cc, np.float64)),
                               _ptr(np.ascontiguousarray(D, np.float64)), _ptr(Ea), _ptr(F))
    return complex(F[0])


def ref_hamiltonian(sysm, kAc, vloc, zproj, dt, zu, ikb_range=None, nthreads=0):
    """Taylor step with the reference AVX stencil (ref_driver.c).  zu is updated
    in place (it must be an aligned array from aligned_state) for orbitals in
    ikb_range (0-based [start, stop)); returns zu."""
    R = ref_lib()
    if R.ref_set_grid(sysm.NLx, sysm.NLy, sysm.NLz) != 0:
        raise ValueError("the reference AVX stencil needs an even NLz")
    d = sysm.desc()
    nkb = sysm.nk_local * sysm.NBoccmax
    s, e = ikb_range if ikb_range is not None else (0, nkb)
    rc = R.ref_hamiltonian(C.byref(d), _ptr(np.ascontiguousarray(kAc, np.float64)), _ptr(np.ascontiguousarray(vloc)),
                           _ptr(zproj), C.c_double(dt), _ptr(zu), C.c_int(s), C.c_int(e), C.c_int(nthreads))
    if rc != 0:
        raise RuntimeError("ref_hamiltonian failed")
    return zu


def aligned_state(zu):
    a = _aligned_complex(zu.shape)
    a[...] = zu
    return a
