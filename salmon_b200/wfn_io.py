"""Ground-state orbital files in SALMON's layout (GS/io_gs_wfn_k.f90:18-62):

  <dir>/gs_wfn_k/occupation             one record: occ(NB, NK), real(8)
  <dir>/gs_wfn_k/wfn_gs_k<ik:07d>.wfn   one record: zu_GS(NL, NB, ik), complex(8)

written with Fortran's unformatted sequential access: each record is framed by
its byte count as a 4-byte little-endian integer before and after the data.
Arrays are column-major (Fortran order), which is the C order of this
package's (nk, NB, NL) and (NK, NB) arrays.  Records of 2^31 bytes or more use
compiler-specific continuation markers and are refused.
"""
from __future__ import annotations

import os

import numpy as np

_MAX_RECORD = 2 ** 31 - 1


def _write_record(path: str, arr: np.ndarray):
    data = np.ascontiguousarray(arr).tobytes()
    if len(data) > _MAX_RECORD:
        raise ValueError(f"{path}: a record of {len(data)} bytes needs continuation markers (not supported)")
    mark = np.array([len(data)], dtype="<i4").tobytes()
    with open(path, "wb") as f:
        f.write(mark)
        f.write(data)
        f.write(mark)


def _read_record(path: str, dtype, count: int) -> np.ndarray:
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 8:
        raise ValueError(f"{path}: not a Fortran unformatted sequential file")
    n = int(np.frombuffer(raw[:4], dtype="<i4")[0])
    if n < 0 or 8 + n > len(raw) or int(np.frombuffer(raw[4 + n:8 + n], dtype="<i4")[0]) != n:
        raise ValueError(f"{path}: record markers do not match (continued or damaged record)")
    want = count * np.dtype(dtype).itemsize
    if n < want:
        raise ValueError(f"{path}: record holds {n} bytes, {want} expected")
    return np.frombuffer(raw[4:4 + want], dtype=dtype).copy()


def gs_wfn_dir(directory: str) -> str:
    return os.path.join(directory, "gs_wfn_k")


def write_gs_wfn_k(directory: str, zu_gs, occ, NK_s: int = 1):
    """Writes occ (NK, NB) and the orbitals zu_gs (nk_local, NB, NL) of k-points
    NK_s..NK_s+nk_local-1 (1-based, as the reference names the files)."""
    d = gs_wfn_dir(directory)
    os.makedirs(d, exist_ok=True)
    _write_record(os.path.join(d, "occupation"), np.asarray(occ, dtype="<f8"))
    zu_gs = np.asarray(zu_gs, dtype="<c16")
    for i in range(zu_gs.shape[0]):
        _write_record(os.path.join(d, f"wfn_gs_k{NK_s + i:07d}.wfn"), zu_gs[i])


def read_gs_wfn_k(directory: str, NK: int, NB: int, NL: int, NK_s: int = 1, NK_e: int | None = None):
    """Reads occ (NK, NB) and the orbitals (NK_e-NK_s+1, NB, NL) of k-points NK_s..NK_e."""
    NK_e = NK if NK_e is None else NK_e
    d = gs_wfn_dir(directory)
    occ = _read_record(os.path.join(d, "occupation"), "<f8", NK * NB).reshape(NK, NB)
    zu = np.empty((NK_e - NK_s + 1, NB, NL), np.complex128)
    for ik in range(NK_s, NK_e + 1):
        zu[ik - NK_s] = _read_record(os.path.join(d, f"wfn_gs_k{ik:07d}.wfn"), "<c16", NB * NL).reshape(NB, NL)
    return zu, occ
