"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute call: this runs without a GPU)."""
import ctypes as C
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(sgpu_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_hot_path():
    names = declared_symbols()
    for required in ("sgpu_create", "sgpu_hamiltonian", "sgpu_hpsi", "sgpu_update_projector", "sgpu_psi_rho",
                     "sgpu_current", "sgpu_energy_terms", "sgpu_set_state", "sgpu_get_state"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from salmon_b200 import build
    path = build.build()
    lib = C.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_abi():
    from salmon_b200 import _lib
    assert set(_lib.ABI) <= set(declared_symbols())


def test_last_error_without_device_call():
    from salmon_b200 import _lib
    msg = _lib.lib().sgpu_last_error()
    assert isinstance(msg, bytes)


def test_create_rejects_bad_descriptor():
    """Argument checks run on the host before any device call."""
    from salmon_b200 import _lib, system as S
    sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=1, nb=2)
    d = sysm.desc()
    d.NBoccmax = d.NB + 1
    h = C.c_void_p()
    rc = _lib.lib().sgpu_create(C.byref(d), 0, C.byref(h))
    assert rc == -1 and not h
    assert b"NBoccmax" in _lib.lib().sgpu_last_error()
    d = sysm.desc()
    rc = _lib.lib().sgpu_create(C.byref(d), 7, C.byref(h))
    assert rc == -1


def test_fortran_binding_names_exist():
    """Every bind(C, name="...") of fortran/salmon_gpu_iface.f90 (the module a
    SALMON maintainer adds; not compiled here) names an entry point the header
    declares and the library exports, and the descriptor type lists the fields
    of sgpu_desc in the header's order."""
    from salmon_b200 import build
    text = open(os.path.join(ROOT, "fortran", "salmon_gpu_iface.f90")).read()
    bound = sorted(set(re.findall(r'bind\(C,\s*name="(sgpu_\w+)"\)', text)))
    assert len(bound) >= 30
    declared = set(declared_symbols())
    lib = C.CDLL(build.build())
    assert [n for n in bound if n not in declared or not hasattr(lib, n)] == []
    ftype = re.search(r"type, bind\(C\) :: sgpu_desc(.*?)end type", text, re.S).group(1)
    fnames = [n.strip().split("(")[0].lower() for line in ftype.splitlines() if "::" in line
              for n in line.split("::")[1].split(",") if n.strip()]
    htext = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "salmon_gpu.h")).read(), flags=re.S)
    hdesc = re.search(r"typedef struct sgpu_desc\s*\{(.*?)\}\s*sgpu_desc;", htext, re.S).group(1)
    hnames = [n.strip().split("[")[0].lower() for decl in hdesc.split(";") if decl.strip()
              for n in re.sub(r"\b(const|int32_t|double|int)\b|\*", " ", decl).split(",") if n.strip()]
    assert fnames == hnames, (fnames, hnames)
