"""ctypes binding of libsalmon_b200.so (include/salmon_gpu.h).

There is no fallback: if the CUDA library is missing or cannot be loaded the
import of the binding raises, and every call that fails on the device raises
SalmonGPUError with the library's message (the reference aborts through
err_finalize, ARTED/main.f90:21-33)."""
from __future__ import annotations

import ctypes as C
import os

from .system import SgpuDesc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsalmon_b200.so")

# symbol -> (restype, argtypes); the list is the ABI of include/salmon_gpu.h
_vp, _dp, _ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
ABI = {
    "sgpu_create": (C.c_int, [C.POINTER(SgpuDesc), _ip, C.POINTER(C.c_void_p)]),
    "sgpu_destroy": (C.c_int, [_vp]),
    "sgpu_set_precision": (C.c_int, [_vp, _ip]),
    "sgpu_last_error": (C.c_char_p, []),
    "sgpu_synchronize": (C.c_int, [_vp]),
    "sgpu_stream": (C.c_void_p, [_vp]),
    "sgpu_set_state": (C.c_int, [_vp, _vp]),
    "sgpu_get_state": (C.c_int, [_vp, _vp]),
    "sgpu_set_state_dev": (C.c_int, [_vp, _vp]),
    "sgpu_state_ptr": (C.c_void_p, [_vp]),
    "sgpu_set_vloc": (C.c_int, [_vp, _vp]),
    "sgpu_set_vpsl": (C.c_int, [_vp, _vp]),
    "sgpu_update_vloc": (C.c_int, [_vp, _vp, _vp]),
    "sgpu_get_vloc": (C.c_int, [_vp, _vp]),
    "sgpu_update_projector": (C.c_int, [_vp, _vp]),
    "sgpu_hamiltonian": (C.c_int, [_vp, C.c_double, _ip]),
    "sgpu_hpsi": (C.c_int, [_vp, _ip, _vp, _vp, _vp]),
    "sgpu_hpsi_batch": (C.c_int, [_vp, _ip, _ip, _vp, _vp]),
    "sgpu_psi_rho": (C.c_int, [_vp, _vp]),
    "sgpu_psi_rho_static": (C.c_int, [_ip, _ip, _ip, _ip, _vp, _vp, _ip, _vp, _vp]),
    "sgpu_current": (C.c_int, [_vp, _vp, _vp]),
    "sgpu_energy_terms": (C.c_int, [_vp, _vp, _dp, _dp]),
    "sgpu_time_kernel": (C.c_int, [_vp, _ip, _ip, _dp]),
    "sgpu_gs_set_state": (C.c_int, [_vp, _vp]),
    "sgpu_gs_get_state": (C.c_int, [_vp, _vp]),
    "sgpu_gram_schmidt": (C.c_int, [_vp]),
    "sgpu_cg": (C.c_int, [_vp, _ip, _vp, _vp]),
    "sgpu_subspace_diag": (C.c_int, [_vp, _vp]),
    "sgpu_gs_to_rt": (C.c_int, [_vp]),
    "sgpu_set_param": (C.c_int, [_vp, _ip, _ip]),
    "sgpu_get_param": (C.c_int, [_vp, _ip, C.POINTER(C.c_int)]),
    "sgpu_cg_residuals": (C.c_int, [_vp, _vp]),
    "sgpu_set_cg_delta": (C.c_int, [_vp, C.c_double]),
    "sgpu_tpa_apply": (C.c_int, [_vp, _vp, _vp, _ip, _vp, _vp]),
    "sgpu_net_weight_count": (C.c_int, []),
    "sgpu_net_set_weights": (C.c_int, [_vp, _vp]),
    "sgpu_net_get_weights": (C.c_int, [_vp, _vp]),
    "sgpu_net_apply": (C.c_int, [_vp, _vp, _vp, _ip]),
    "sgpu_net_grad": (C.c_int, [_vp, _vp, _vp, _ip, _vp, _dp]),
    "sgpu_net_train_step": (C.c_int, [_vp, _vp, _vp, _ip, C.c_float, _dp]),
    "sgpu_autotune": (C.c_int, [_vp, _ip, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
    "sgpu_vloc_history_reset": (C.c_int, [_vp]),
    "sgpu_vloc_extrapolate": (C.c_int, [_vp]),
    "sgpu_check_desc": (C.c_int, [_vp]),
    "sgpu_psi_rho_dev": (C.c_int, [_vp, _vp]),
    "sgpu_current_dev": (C.c_int, [_vp, _vp, _vp]),
    "sgpu_update_vloc_dev": (C.c_int, [_vp, _vp, _vp]),
    "sgpu_autotune_step": (C.c_int, [_vp, C.c_double, _ip, C.POINTER(C.c_int), _dp]),
    "sgpu_batch_create": (C.c_int, [C.POINTER(C.c_void_p), _ip, C.POINTER(C.c_void_p)]),
    "sgpu_batch_step": (C.c_int, [_vp, _vp, _ip]),
    "sgpu_batch_stream": (C.c_void_p, [_vp]),
    "sgpu_batch_destroy": (C.c_int, [_vp]),
}

PARAMS = {"nslab": 0, "launches": 1, "uvpsi_split": 2, "cg_precond": 3, "pass_tables": 4, "kb_kernel": 5,
          "pass_fixed": 6, "cur_fixed": 7, "taylor_kernel": 8, "nsp": 9,
          "kb_split": 10}

KERNELS = {"stencil_pass": 0, "taylor_stage": 1, "taylor_last": 1, "uvpsi": 2, "psi_rho": 3, "kb_field": 4, "kb_term": 5,
           "current_stencil": 6, "current_proj": 7}

_LIB = None


class SalmonGPUError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, call, code, msg):
        super().__init__(f"{call} failed ({code}): {msg}")
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run `python -m salmon_b200.build` "
                               "(the CUDA library is required; there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in ABI.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(name, rc):
    if rc != 0:
        raise SalmonGPUError(name, rc, lib().sgpu_last_error().decode())
    return rc


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))
