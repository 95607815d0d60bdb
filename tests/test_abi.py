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
