"""Host-side mirror of SALMON's RT hot-path routines over the C ABI.

The methods keep the reference's names and argument meaning (paths relative to
the SALMON source tree):

  update_projector(kAc)        common/projector.f90:29      zproj for k+A(t)
  hamiltonian(dt)              RT/hamiltonian.f90:27         4th-order Taylor step
  hpsi_omp_KB_RT(ik, tpsi)     common/hpsi.f90:89            H psi, one orbital
  hpsi_omp_KB_GS(ik, tpsi)     common/hpsi.f90:33            H psi and H psi - V psi
  psi_rho_RT()                 common/psi_rho.f90:40         density (before allreduce)
  current_RT(kAc)              RT/current.f90:65             current (before allreduce)
  energy_terms(kAc)            common/total_energy.f90:113   Ekin, Enl

Orbitals stay on the device between calls; numpy arrays follow
salmon_b200.system conventions: zu is complex128 of shape (nk_local, NBoccmax, NL).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SalmonGPUError, call

PRECISIONS = {"c128": 0, "c64": 1}


def _vp(a):
    return C.c_void_p(a.ctypes.data)


class GpuSystem:
    """One handle of the CUDA library: a system's tables plus its resident orbitals."""

    def __init__(self, sysm, precision: str = "c128"):
        self.sysm = sysm
        self._desc = sysm.desc()
        self._h = C.c_void_p()
        call("sgpu_create", C.byref(self._desc), PRECISIONS[precision], C.byref(self._h))
        self.precision = precision

    # ---- lifetime
    def close(self):
        if self._h:
            _lib.lib().sgpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return _lib.lib().sgpu_stream(self._h) or 0

    def state_ptr(self) -> int:
        return _lib.lib().sgpu_state_ptr(self._h) or 0

    def synchronize(self):
        call("sgpu_synchronize", self._h)

    def set_precision(self, precision: str):
        call("sgpu_set_precision", self._h, PRECISIONS[precision])
        self.precision = precision

    # ---- resident state
    def set_state(self, zu):
        s = self.sysm
        zu = np.ascontiguousarray(zu, dtype=np.complex128)
        if zu.shape != (s.nk_local, s.NBoccmax, s.NL):
            raise ValueError(f"zu must have shape {(s.nk_local, s.NBoccmax, s.NL)}, got {zu.shape}")
        call("sgpu_set_state", self._h, _vp(zu))

    def set_state_dev(self, zu_dev: int):
        """Resident orbitals from a device complex(8) array zu(NL,NBoccmax,NK_s:NK_e)."""
        call("sgpu_set_state_dev", self._h, C.c_void_p(zu_dev))

    def get_state(self):
        s = self.sysm
        zu = np.empty((s.nk_local, s.NBoccmax, s.NL), np.complex128)
        call("sgpu_get_state", self._h, _vp(zu))
        return zu

    def set_vloc(self, vloc):
        v = np.ascontiguousarray(vloc, dtype=np.float64)
        if v.shape != (self.sysm.NL,):
            raise ValueError("Vloc must have shape (NL,)")
        call("sgpu_set_vloc", self._h, _vp(v))

    # ---- hot path
    def set_vpsl(self, vpsl):
        v = np.ascontiguousarray(vpsl, dtype=np.float64)
        call("sgpu_set_vpsl", self._h, _vp(v))

    def update_vloc(self, rho=None):
        """Vloc = Vh[rho] + Vpsl + Vexc[rho] on the device (Hartree + PZ LDA);
        rho defaults to the resident orbitals' density.  Returns (Eh, Exc)."""
        e = np.zeros(2)
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        call("sgpu_update_vloc", self._h, None if r is None else _vp(r), _vp(e))
        return float(e[0]), float(e[1])

    def vloc_history_reset(self):
        """Vloc_old(:,1) = Vloc_old(:,2) = Vloc (control_sc.f90:82), for the etrs propagator."""
        call("sgpu_vloc_history_reset", self._h)

    def vloc_extrapolate(self):
        """Vloc <- 3 Vloc - 3 Vloc_old(:,1) + Vloc_old(:,2), history shifted (dt_evolve.f90:248-252)."""
        call("sgpu_vloc_extrapolate", self._h)

    def get_vloc(self):
        v = np.empty(self.sysm.NL)
        call("sgpu_get_vloc", self._h, _vp(v))
        return v

    def update_projector(self, kAc):
        k = np.ascontiguousarray(kAc, dtype=np.float64)
        if k.shape != (3, self.sysm.NK):
            raise ValueError("kAc must have shape (3, NK) (Fortran kAc(NK,3))")
        call("sgpu_update_projector", self._h, _vp(k))

    def hamiltonian(self, dt: float, flag_current: bool = False):
        call("sgpu_hamiltonian", self._h, C.c_double(dt), int(flag_current))

    def hpsi_omp_KB_RT(self, ik: int, tpsi):
        t = np.ascontiguousarray(tpsi, dtype=np.complex128)
        h = np.empty_like(t)
        call("sgpu_hpsi", self._h, ik, _vp(t), _vp(h), None)
        return h

    def hpsi_omp_KB_GS(self, ik: int, tpsi):
        t = np.ascontiguousarray(tpsi, dtype=np.complex128)
        h = np.empty_like(t)
        tt = np.empty_like(t)
        call("sgpu_hpsi", self._h, ik, _vp(t), _vp(h), _vp(tt))
        return h, tt

    def hpsi_batch(self, ikb_s: int, ikb_e: int, tpsi_dev: int, htpsi_dev: int):
        call("sgpu_hpsi_batch", self._h, ikb_s, ikb_e, C.c_void_p(tpsi_dev), C.c_void_p(htpsi_dev))

    def set_param(self, name: str, value: int):
        call("sgpu_set_param", self._h, _lib.PARAMS[name], int(value))

    def get_param(self, name: str) -> int:
        v = C.c_int()
        call("sgpu_get_param", self._h, _lib.PARAMS[name], C.byref(v))
        return v.value

    def autotune(self, reps: int = 5):
        """Times every launch shape the library knows on the resident orbitals and
        keeps the fastest; returns (nslab, uvpsi_split, ms per H application)."""
        ns, sp, ms = C.c_int(), C.c_int(), C.c_double()
        call("sgpu_autotune", self._h, int(reps), C.byref(ns), C.byref(sp), C.byref(ms))
        return ns.value, sp.value, ms.value

    TUNE_PARAMS = ("taylor_kernel", "pass_fixed", "pass_tables", "nslab", "kb_kernel", "uvpsi_split")

    def autotune_step(self, dt: float = 0.02, reps: int = 3):
        """Times whole Taylor steps for every launch choice (sgpu_autotune_step),
        keeps the fastest; returns ({param: value}, ms per step)."""
        p = (C.c_int * 6)()
        ms = C.c_double()
        call("sgpu_autotune_step", self._h, C.c_double(dt), int(reps), p, C.byref(ms))
        return dict(zip(self.TUNE_PARAMS, list(p))), ms.value

    def get_nsp(self) -> int:
        """Sphere points of the handle (the union of the projectors' points)."""
        v = C.c_int()
        call("sgpu_get_param", self._h, _lib.PARAMS["nsp"], C.byref(v))
        return v.value

    def time_kernel(self, kernel: str, reps: int = 10) -> float:
        """Mean device milliseconds per launch of one library kernel (CUDA events on the library stream)."""
        ms = C.c_double()
        call("sgpu_time_kernel", self._h, _lib.KERNELS[kernel], reps, C.byref(ms))
        return ms.value

    # ---- ground state (FP64)
    def gs_set_state(self, zu_gs):
        s = self.sysm
        z = np.ascontiguousarray(zu_gs, dtype=np.complex128)
        if z.shape != (s.nk_local, s.NB, s.NL):
            raise ValueError(f"zu_GS must have shape {(s.nk_local, s.NB, s.NL)}")
        call("sgpu_gs_set_state", self._h, _vp(z))

    def gs_get_state(self):
        s = self.sysm
        z = np.empty((s.nk_local, s.NB, s.NL), np.complex128)
        call("sgpu_gs_get_state", self._h, _vp(z))
        return z

    def gram_schmidt(self):
        """Gram_Schmidt_ompk (GS/Gram_Schmidt.f90:32-55) on the device ground-state orbitals."""
        call("sgpu_gram_schmidt", self._h)

    def cg(self, ncg: int):
        """CG_ompk (GS/CG.f90:34-139); returns (esp_var (nkl,NB), iterations (nkl,NB))."""
        s = self.sysm
        esp = np.empty((s.nk_local, s.NB))
        its = np.empty((s.nk_local, s.NB), np.int32)
        call("sgpu_cg", self._h, int(ncg), _vp(esp), _vp(its))
        return esp, its

    def subspace_diag(self):
        """diag_omp (GS/diag.f90:22-173); returns the eigenvalues esp (nkl,NB)."""
        s = self.sysm
        esp = np.empty((s.nk_local, s.NB))
        call("sgpu_subspace_diag", self._h, _vp(esp))
        return esp

    def gs_to_rt(self):
        call("sgpu_gs_to_rt", self._h)

    def cg_residuals(self):
        """Residual norms (nkl, NB) of every band after the last ``cg`` (no occupation factor)."""
        s = self.sysm
        r = np.empty((s.nk_local, s.NB))
        call("sgpu_cg_residuals", self._h, _vp(r))
        return r

    def set_cg_delta(self, delta_cg: float):
        """Per-band CG stopping threshold on the Rayleigh quotient (reference: 1e-15)."""
        call("sgpu_set_cg_delta", self._h, C.c_double(delta_cg))

    def set_cg_preconditioner(self, kind: str):
        """'plain' (the reference's CG), 'tpa' or 'learned' (needs ``net_set_weights``)."""
        self.set_param("cg_precond", {"plain": 0, "tpa": 1, "learned": 2}[kind])

    def tpa_apply(self, in_dev: int, out_dev: int, nvec: int, tband, kidx=None):
        """TPA on nvec device vectors; vector v at local k-point kidx[v] (default v)."""
        tb = np.ascontiguousarray(tband, dtype=np.float64)
        kv = None if kidx is None else np.ascontiguousarray(kidx, dtype=np.int32)
        call("sgpu_tpa_apply", self._h, C.c_void_p(in_dev), C.c_void_p(out_dev), int(nvec),
             None if kv is None else _vp(kv), _vp(tb))

    # ---- learned preconditioner
    @staticmethod
    def net_weight_count() -> int:
        return _lib.lib().sgpu_net_weight_count()

    def net_set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != self.net_weight_count():
            raise ValueError(f"need {self.net_weight_count()} weights")
        call("sgpu_net_set_weights", self._h, _vp(w))

    def net_get_weights(self):
        w = np.empty(self.net_weight_count(), np.float32)
        call("sgpu_net_get_weights", self._h, _vp(w))
        return w

    def net_apply(self, in_dev: int, out_dev: int, nvec: int):
        call("sgpu_net_apply", self._h, C.c_void_p(in_dev), C.c_void_p(out_dev), int(nvec))

    def net_grad(self, g_dev: int, t_dev: int, nvec: int):
        grad = np.empty(self.net_weight_count(), np.float32)
        loss = C.c_double()
        call("sgpu_net_grad", self._h, C.c_void_p(g_dev), C.c_void_p(t_dev), int(nvec), _vp(grad), C.byref(loss))
        return grad, loss.value

    def net_train_step(self, g_dev: int, t_dev: int, nvec: int, lr: float) -> float:
        loss = C.c_double()
        call("sgpu_net_train_step", self._h, C.c_void_p(g_dev), C.c_void_p(t_dev), int(nvec), C.c_float(lr),
             C.byref(loss))
        return loss.value

    # ---- reductions
    def psi_rho_RT(self):
        rho = np.empty(self.sysm.NL)
        call("sgpu_psi_rho", self._h, _vp(rho))
        return rho

    def psi_rho_dev(self, rho_dev: int):
        """rho(NL) of the resident orbitals into the DEV FP64 buffer at rho_dev,
        enqueued on the handle's stream (not waited for)."""
        call("sgpu_psi_rho_dev", self._h, C.c_void_p(rho_dev))

    def current_dev(self, kAc, jav_dev: int):
        """J(3) at kAc into the DEV FP64 buffer at jav_dev, on the handle's stream."""
        k = np.ascontiguousarray(np.asarray(kAc, dtype=np.float64))
        call("sgpu_current_dev", self._h, _vp(k), C.c_void_p(jav_dev))

    def update_vloc_dev(self, rho_dev: int, eh_exc_dev: int = 0):
        """Vloc = Vh + Vpsl + Vexc from the DEV density at rho_dev, on the handle's stream."""
        call("sgpu_update_vloc_dev", self._h, C.c_void_p(rho_dev), C.c_void_p(eh_exc_dev or None))

    def current_RT(self, kAc):
        k = np.ascontiguousarray(kAc, dtype=np.float64)
        jav = np.empty(3)
        call("sgpu_current", self._h, _vp(k), _vp(jav))
        return jav

    def energy_terms(self, kAc):
        k = np.ascontiguousarray(kAc, dtype=np.float64)
        ek, en = C.c_double(), C.c_double()
        call("sgpu_energy_terms", self._h, _vp(k), C.byref(ek), C.byref(en))
        return ek.value, en.value


def check_desc(sysm) -> None:
    """The descriptor checks of sgpu_create on the host (no device call);
    raises SalmonGPUError with the library's reason."""
    d = sysm.desc()
    call("sgpu_check_desc", C.byref(d))


class GpuBatch:
    """Several GpuSystem handles advanced together, one CUDA-graph replay per call
    of ``step`` (sgpu_batch_*)."""

    def __init__(self, systems):
        self.systems = list(systems)
        arr = (C.c_void_p * len(self.systems))(*[g.handle for g in self.systems])
        self._b = C.c_void_p()
        call("sgpu_batch_create", arr, len(self.systems), C.byref(self._b))

    def step(self, dts, nsteps: int = 1):
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float64), (len(self.systems),)))
        call("sgpu_batch_step", self._b, _vp(d), int(nsteps))

    @property
    def stream(self) -> int:
        return _lib.lib().sgpu_batch_stream(self._b) or 0

    def close(self):
        if self._b:
            call("sgpu_batch_destroy", self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


__all__ = ["GpuSystem", "GpuBatch", "SalmonGPUError", "PRECISIONS", "check_desc"]
