"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (max |gpu - oracle| / max |oracle|):
  complex(8) path:  1e-12 for H psi, the Taylor step and every FP64 reduction
  complex(4) path:  H psi 2e-6, one Taylor step 2e-6 (FP32 orbitals and stencil);
                    reductions of the complex(4) orbitals 1e-12 against the oracle
                    run on the same rounded orbitals (they accumulate in FP64)
"""
import numpy as np
import pytest

from _helpers import grid_system, rel
from oracle import oracle as O
from salmon_b200 import system as S

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32_HPSI = 2e-6
TOL32_STEP = 2e-6

CASES = {
    "ragged_even_z": lambda: S.small_system(8, 10, 12, nk=3, nb=4, seed=21),
    "ragged_odd_z": lambda: S.small_system(9, 8, 11, nk=2, nb=3, seed=22),
    "microbench_20": lambda: S.microbench_system(20, nk_limit=2, Nb=32),
    "microbench_16": lambda: S.microbench_system(16, nk_limit=1, Nb=32),
    # planes wider than one CTA (NLy*NLz/2 > 512): the pass splits them into y-blocks
    "wide_48": lambda: S.microbench_system(48, nk_limit=1, Nb=4),
    # the compile-time 32x32 forms of the pass and of the current stencil
    "microbench_32": lambda: S.microbench_system(32, nk_limit=1, Nb=4),
    "wide_ragged": lambda: S.small_system(6, 50, 22, nk=2, nb=3, a=(5.0, 12.0, 9.0), seed=23),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, cuda_lib):
    sysm, kAc, vloc, zu = CASES[request.param]()
    _, zproj = O.update_projector(sysm, kAc)
    return request.param, sysm, kAc, vloc, zu, zproj


def make_gpu(sysm, kAc, vloc, zu, precision="c128"):
    from salmon_b200.rt import GpuSystem
    g = GpuSystem(sysm, precision)
    g.set_state(zu)
    g.set_vloc(vloc)
    g.update_projector(kAc)
    return g


def c64_round(z):
    return z.astype(np.complex64).astype(np.complex128)


def test_state_round_trip(case):
    _, sysm, kAc, vloc, zu, _ = case
    with make_gpu(sysm, kAc, vloc, zu) as g:
        np.testing.assert_array_equal(g.get_state(), zu)
    with make_gpu(sysm, kAc, vloc, zu, "c64") as g:
        np.testing.assert_array_equal(g.get_state(), c64_round(zu))


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_hpsi_matches_oracle(case, precision):
    _, sysm, kAc, vloc, zu, zproj = case
    tol = TOL64 if precision == "c128" else TOL32_HPSI
    with make_gpu(sysm, kAc, vloc, zu, precision) as g:
        for ikl in range(sysm.nk_local):
            ik = sysm.NK_s + ikl
            t = zu[ikl, -1]
            h_ref, tt_ref = O.hpsi(sysm, kAc, vloc, zproj, ik, t, want_tt=True)
            h = g.hpsi_omp_KB_RT(ik, t)
            assert rel(h, h_ref) < tol
            h2, tt = g.hpsi_omp_KB_GS(ik, t)
            assert rel(h2, h_ref) < tol
            assert rel(tt, tt_ref) < tol


def test_taylor_step_c128(case):
    _, sysm, kAc, vloc, zu, zproj = case
    dt = 0.08
    with make_gpu(sysm, kAc, vloc, zu) as g:
        g.hamiltonian(dt)
        z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, dt, zu)
        assert rel(g.get_state(), z_ref) < TOL64
        # two more steps at a new k+A(t), as dt_evolve does (update_projector, then hamiltonian)
        k2 = kAc + np.array([0.0, 0.0, 2e-3])[:, None]
        _, zp2 = O.update_projector(sysm, k2)
        g.update_projector(k2)
        g.hamiltonian(dt)
        g.hamiltonian(dt)
        z_ref = O.hamiltonian(sysm, k2, vloc, zp2, dt, O.hamiltonian(sysm, k2, vloc, zp2, dt, z_ref))
        assert rel(g.get_state(), z_ref) < TOL64


def test_taylor_step_c64(case):
    _, sysm, kAc, vloc, zu, zproj = case
    dt = 0.08
    with make_gpu(sysm, kAc, vloc, zu, "c64") as g:
        g.hamiltonian(dt)
        z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, dt, c64_round(zu))
        assert rel(g.get_state(), z_ref) < TOL32_STEP


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_reductions_fp64(case, precision):
    _, sysm, kAc, vloc, zu, _ = case
    z_in = zu if precision == "c128" else c64_round(zu)
    kcur = kAc + np.array([0.0, 1e-3, 0.0])[:, None]
    with make_gpu(sysm, kAc, vloc, zu, precision) as g:
        assert rel(g.psi_rho_RT(), O.psi_rho(sysm, z_in)) < TOL64
        assert rel(g.current_RT(kcur), O.current(sysm, kcur, z_in)) < TOL64
        ek, en = g.energy_terms(kcur)
        ek_ref, en_ref = O.energy_terms(sysm, kcur, z_in)
        assert abs(ek - ek_ref) < TOL64 * abs(ek_ref)
        assert abs(en - en_ref) < TOL64 * max(abs(en_ref), 1e-300)


def test_hpsi_batch_device_pointers(case):
    import torch
    _, sysm, kAc, vloc, zu, zproj = case
    with make_gpu(sysm, kAc, vloc, zu) as g:
        nb = min(5, sysm.nk_local * sysm.NBoccmax)
        src = torch.from_numpy(zu.reshape(-1, sysm.NL)[:nb].copy()).cuda()
        dst = torch.empty_like(src)
        torch.cuda.synchronize()
        g.hpsi_batch(1, nb, src.data_ptr(), dst.data_ptr())
        g.synchronize()
        out = dst.cpu().numpy()
        for o in range(nb):
            ik = sysm.NK_s + o // sysm.NBoccmax
            assert rel(out[o], O.hpsi(sysm, kAc, vloc, zproj, ik, zu.reshape(-1, sysm.NL)[o])) < TOL64


def test_no_projectors(cuda_lib):
    """NI = 0: the stencil alone (the reference's stencilperf configuration, Nlma=0)."""
    sysm = grid_system((10, 12, 8), nk=2, nb=3)
    sysm.kAc0 = np.array([[0.1, -0.2], [0.05, 0.0], [0.3, 0.1]])
    rng = np.random.default_rng(0)
    zu = rng.standard_normal((2, 3, sysm.NL)) + 1j * rng.standard_normal((2, 3, sysm.NL))
    vloc = rng.uniform(-1, 0, sysm.NL)
    kAc = sysm.kAc0
    _, zproj = O.update_projector(sysm, kAc)
    with make_gpu(sysm, kAc, vloc, zu) as g:
        g.hamiltonian(0.05)
        assert rel(g.get_state(), O.hamiltonian(sysm, kAc, vloc, zproj, 0.05, zu)) < TOL64


def test_precision_switch_keeps_state(cuda_lib):
    sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=1, nb=2, seed=9)
    with make_gpu(sysm, kAc, vloc, zu) as g:
        g.set_precision("c64")
        np.testing.assert_array_equal(g.get_state(), c64_round(zu))
        g.set_precision("c128")
        np.testing.assert_array_equal(g.get_state(), c64_round(zu))


def test_errors_are_reported_not_fatal(cuda_lib):
    from salmon_b200.rt import GpuSystem, SalmonGPUError
    sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=1, nb=2, seed=9)
    with GpuSystem(sysm) as g:
        with pytest.raises(SalmonGPUError, match="state, Vloc and projectors"):
            g.hamiltonian(0.1)
        g.set_vloc(vloc)
        g.update_projector(kAc)
        with pytest.raises(SalmonGPUError, match="ik outside"):
            g.hpsi_omp_KB_RT(5, zu[0, 0])


@pytest.mark.parametrize("nslab", [1, 3])
@pytest.mark.parametrize("tables", [0, 1])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_pass_table_staging(case, precision, tables, nslab):
    """The stencil pass with Vloc and the sphere-index table staged through
    shared memory (or loaded from global memory one plane ahead), with the
    orbitals split into x-slabs: H psi, the GS form and a Taylor step against the oracle."""
    _, sysm, kAc, vloc, zu, zproj = case
    dt = 0.08
    tol_h, tol_s = (TOL64, TOL64) if precision == "c128" else (TOL32_HPSI, TOL32_STEP)
    z0 = zu if precision == "c128" else c64_round(zu)
    with make_gpu(sysm, kAc, vloc, zu, precision) as g:
        g.set_param("pass_tables", tables)
        g.set_param("nslab", min(nslab, sysm.NLx))
        assert g.get_param("pass_tables") == tables
        ik = sysm.NK_s
        t = zu[0, -1]
        h_ref, tt_ref = O.hpsi(sysm, kAc, vloc, zproj, ik, t, want_tt=True)
        assert rel(g.hpsi_omp_KB_RT(ik, t), h_ref) < tol_h
        h2, tt = g.hpsi_omp_KB_GS(ik, t)
        assert rel(h2, h_ref) < tol_h and rel(tt, tt_ref) < tol_h
        g.hamiltonian(dt)
        assert rel(g.get_state(), O.hamiltonian(sysm, kAc, vloc, zproj, dt, z0)) < tol_s


# KB term forms: the band-group tile kernel, the band-quad kernel with 4 warps a
# quad, and the split form: the tile kernel's projections over 1 or 3 point ranges
# followed by the field kernel
KB_FORMS = {"tile": {"kb_kernel": 1}, "quad4": {"kb_kernel": 2, "uvpsi_split": 4},
            "split1": {"kb_kernel": 3, "kb_split": 1}, "split3": {"kb_kernel": 3, "kb_split": 3}}


def _kb_form_checks(sysm, kAc, vloc, zu, zproj, precision, form):
    import torch
    tol_h, tol_s = (TOL64, TOL64) if precision == "c128" else (TOL32_HPSI, TOL32_STEP)
    z0 = zu if precision == "c128" else c64_round(zu)
    with make_gpu(sysm, kAc, vloc, zu, precision) as g:
        for k, v in KB_FORMS[form].items():
            g.set_param(k, v)
            assert g.get_param(k) == v
        for ikl in range(sysm.nk_local):
            ik = sysm.NK_s + ikl
            t = zu[ikl, -1]
            assert rel(g.hpsi_omp_KB_RT(ik, t), O.hpsi(sysm, kAc, vloc, zproj, ik, t)) < tol_h
        if precision == "c128":  # a band range that starts and ends inside k-point blocks
            flat = zu.reshape(-1, sysm.NL)
            o0, nb = 1, min(flat.shape[0] - 1, sysm.NBoccmax + 3)
            src = torch.from_numpy(flat[o0:o0 + nb].copy()).cuda()
            dst = torch.empty_like(src)
            torch.cuda.synchronize()
            g.hpsi_batch(o0 + 1, o0 + nb, src.data_ptr(), dst.data_ptr())  # 1-based, inclusive
            g.synchronize()
            out = dst.cpu().numpy()
            for i in range(nb):
                o = o0 + i
                ik = sysm.NK_s + o // sysm.NBoccmax
                assert rel(out[i], O.hpsi(sysm, kAc, vloc, zproj, ik, flat[o])) < tol_h
        g.hamiltonian(0.08)
        assert rel(g.get_state(), O.hamiltonian(sysm, kAc, vloc, zproj, 0.08, z0)) < tol_s


@pytest.mark.parametrize("form", list(KB_FORMS))
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_kb_forms(case, precision, form):
    """The KB term of H psi by each form (KB_FORMS): single orbitals, a band range
    that cuts k-point blocks, and a Taylor step, against the oracle."""
    _, sysm, kAc, vloc, zu, zproj = case
    _kb_form_checks(sysm, kAc, vloc, zu, zproj, precision, form)


@pytest.mark.parametrize("form", list(KB_FORMS))
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_kb_forms_many_bands(cuda_lib, precision, form):
    """More bands than one tile's 32 (a partial second band group) and three
    atoms whose spheres overlap."""
    sysm, kAc, vloc, zu = S.small_system(8, 10, 12, nk=2, nb=37, nat=3, seed=31, Rps=2.2)
    _, zproj = O.update_projector(sysm, kAc)
    _kb_form_checks(sysm, kAc, vloc, zu, zproj, precision, form)


@pytest.mark.parametrize("kb_kernel", [1, 3])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_kb_tile_32cubed(cuda_lib, precision, kb_kernel):
    """The band-group KB kernel and its split form at a production grid (32^3, 8
    atoms, ~1000 points per sphere: the largest shared-memory tile) against the oracle."""
    sysm, kAc, vloc, zu = S.microbench_system(32, nk_limit=1, Nb=8)
    _, zproj = O.update_projector(sysm, kAc)
    tol = TOL64 if precision == "c128" else TOL32_HPSI
    with make_gpu(sysm, kAc, vloc, zu, precision) as g:
        g.set_param("kb_kernel", kb_kernel)
        ik = sysm.NK_s
        for b in (0, sysm.NBoccmax - 1):
            t = zu[0, b]
            assert rel(g.hpsi_omp_KB_RT(ik, t), O.hpsi(sysm, kAc, vloc, zproj, ik, t)) < tol
