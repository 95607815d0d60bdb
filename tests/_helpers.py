"""Shared helpers for the tests (not collected)."""
import os

import numpy as np

from salmon_b200 import system as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def system_from_arrays(g):
    """Rebuilds a System from arrays stored by tests/golden/make_golden.py."""
    nl = g["NL"]
    nb = g["NB"]
    return S.System(NLx=int(nl[0]), NLy=int(nl[1]), NLz=int(nl[2]), aL=g["aL"], kAc0=g["kAc0"], NB=int(nb[0]),
                    NBoccmax=int(nb[1]), occ=g["occ"], Rion=g["Rion"], Rps=float(g["Rps"]), Mps=g["Mps"],
                    Jxyz=g["Jxyz"], Jxx=g["Jxx"], Jyy=g["Jyy"], Jzz=g["Jzz"], uV=g["uV"], iuV=g["iuV"],
                    a_tbl=g["a_tbl"])


def grid_system(shape, aL=(6.0, 6.5, 7.0), nk=1, nb=1):
    """A system without projectors (NI=0): just the grid, k-points and occupations."""
    z = np.zeros((0, 1), np.int32)
    return S.System(NLx=shape[0], NLy=shape[1], NLz=shape[2], aL=np.asarray(aL, float),
                    kAc0=np.zeros((3, nk)), NB=nb, NBoccmax=nb, occ=np.ones((nk, nb)), Rion=np.zeros((0, 3)),
                    Rps=1.0, Mps=np.zeros(0, np.int32), Jxyz=z, Jxx=z, Jyy=z, Jzz=z, uV=np.zeros((0, 1)),
                    iuV=np.zeros(0, np.int32), a_tbl=np.zeros(0, np.int32))


def coefs(sysm, k):
    ln = sysm.lap_nab()
    lapt = np.concatenate([ln["lapx"][1:], ln["lapy"][1:], ln["lapz"][1:]])
    nab = np.concatenate([ln["nabx"][1:], ln["naby"][1:], ln["nabz"][1:]])
    nabt = np.concatenate([k[0] * ln["nabx"][1:], k[1] * ln["naby"][1:], k[2] * ln["nabz"][1:]])
    A = (k @ k - (ln["lapx"][0] + ln["lapy"][0] + ln["lapz"][0])) * 0.5
    return lapt, nab, nabt, A


def rel(a, b):
    """max |a-b| / max |b|"""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
