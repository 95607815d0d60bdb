"""sgpu_psi_rho_static (static device scratch, no allocation) against the
handle's sgpu_psi_rho on the same orbitals.

Collected last so that it also runs after every other GPU test in one process;
it passes on its own in a fresh process too.  Tolerance: 1e-12 relative to
max(rho) (both are FP64 reductions in the same orbital order)."""
import ctypes as C

import numpy as np
import pytest

from salmon_b200 import _lib, system as S

MAX = 2097152  # SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES


def _static(prec, NL, nb, nk, zu, occ, ld_occ, rho, stream):
    return _lib.lib().sgpu_psi_rho_static(prec, NL, nb, nk, C.c_void_p(zu), C.c_void_p(occ), ld_occ,
                                          C.c_void_p(rho), C.c_void_p(stream))


def test_rejects_bad_arguments_before_any_device_call():
    """Host-side checks; these calls reach no CUDA function."""
    fake = 1 << 20  # aligned, never dereferenced
    assert _static(0, 1 << 22, 1, 1, fake, fake, 1, fake, 0) == -1       # 4M doubles > maximum
    assert b"static maximum" in _lib.lib().sgpu_last_error()
    assert _static(0, 32768, 64, 65, fake, fake, 64, fake, 0) == -1      # 65 chunks x 32768 > maximum
    assert _static(0, 16, 4, 2, fake, fake, 3, fake, 0) == -1            # ld_occ < nb
    assert _static(5, 16, 4, 2, fake, fake, 4, fake, 0) == -1            # precision
    assert _static(0, 16, 4, 2, fake + 8, fake, 4, fake, 0) == -1        # complex(8) needs 16-byte alignment
    assert _static(0, 16, 4, 2, 0, fake, 4, fake, 0) == -1               # null


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ragged", "microbench16"])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_static_scratch_matches_handle(cuda_lib, case, precision):
    import torch
    from salmon_b200.rt import GpuSystem, PRECISIONS
    if case == "ragged":
        sysm, kAc, vloc, zu = S.small_system(8, 9, 10, nk=3, nb=5)
    else:
        sysm, kAc, vloc, zu = S.microbench_system(16, nkgrid=(2, 2, 2), Nb=8)
    NL, nb, nk = sysm.NL, sysm.NBoccmax, sysm.nk_local
    with GpuSystem(sysm, precision) as g:
        g.set_state(zu)
        rho_ref = g.psi_rho_RT()
        occ = torch.from_numpy(np.ascontiguousarray(sysm.occ, dtype=np.float64).ravel()).cuda()  # occ(NB,NK)
        rho = torch.empty(NL, dtype=torch.float64, device="cuda")
        for call in range(2):
            rho.fill_(float("nan"))
            torch.cuda.synchronize()
            rc = _static(PRECISIONS[precision], NL, nb, nk, g.state_ptr(), occ.data_ptr(), sysm.NB,
                         rho.data_ptr(), g.stream)
            assert rc == 0, _lib.lib().sgpu_last_error()
            g.synchronize()
            got = rho.cpu().numpy()
            err = np.abs(got - rho_ref).max() / np.abs(rho_ref).max()
            assert err <= 1e-12, (call, err)


def _rho_numpy(zu, occ_nb_nk):
    """rho = sum_{k,b} occ(b,k) |zu(:,b,k)|^2 in FP64 (zu as [nk][nb][NL])."""
    z = np.asarray(zu, dtype=np.complex128)
    return np.einsum("kb,kbi->i", occ_nb_nk, (z.real ** 2 + z.imag ** 2))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_static_scratch_many_chunks(cuda_lib, precision):
    """nb*nk = 185 orbitals: three partial-density rows (grid.y = 3), the last
    one partial, summed by k_rho_sum_static; checked against an independent
    NumPy sum with occupations that differ per orbital."""
    import torch
    from salmon_b200.rt import GpuSystem, PRECISIONS
    sysm, kAc, vloc, zu = S.small_system(8, 9, 10, nk=5, nb=37, seed=31)
    NL, nb, nk = sysm.NL, sysm.NBoccmax, sysm.nk_local
    assert nb * nk > 128 and (nb * nk) % 64 != 0
    occ_h = np.random.default_rng(5).uniform(0.1, 2.0, size=(nk, nb))   # C order [k][b] = Fortran occ(NB,NK)
    z_in = zu if precision == "c128" else zu.astype(np.complex64)
    ref = _rho_numpy(z_in, occ_h)
    with GpuSystem(sysm, precision) as g:
        g.set_state(zu)
        occ = torch.from_numpy(occ_h.ravel().copy()).cuda()
        rho = torch.empty(NL, dtype=torch.float64, device="cuda")
        for call in range(2):
            rho.fill_(float("nan"))
            torch.cuda.synchronize()
            rc = _static(PRECISIONS[precision], NL, nb, nk, g.state_ptr(), occ.data_ptr(), nb, rho.data_ptr(),
                         g.stream)
            assert rc == 0, _lib.lib().sgpu_last_error()
            g.synchronize()
            got = rho.cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), call


@pytest.mark.gpu
def test_static_scratch_at_capacity_allocates_nothing(cuda_lib):
    """The largest accepted problem: ceil(nb*nk/64) * NL equals the static
    maximum exactly (NL = 1024, 2048 partial rows, 131040 complex(4) orbitals,
    1.07 GB).  One orbital more is rejected.  After a first call, a second call
    leaves the device's free memory unchanged: the entry point allocates
    nothing."""
    import torch
    NL, nb, nk = 1024, 40, 3276
    norb = nb * nk
    assert -(-norb // 64) * NL == MAX
    gen = torch.Generator(device="cuda").manual_seed(7)
    zu = torch.randn(norb, NL, dtype=torch.complex64, device="cuda", generator=gen)
    occ = torch.rand(norb, dtype=torch.float64, device="cuda", generator=gen) + 0.5
    rho = torch.empty(NL, dtype=torch.float64, device="cuda")
    ref = torch.zeros(NL, dtype=torch.float64, device="cuda")
    for o0 in range(0, norb, 8192):  # FP64 reference in slices (keeps the check's own memory small)
        z = zu[o0:o0 + 8192].to(torch.complex128)
        ref += (occ[o0:o0 + 8192, None] * (z.real ** 2 + z.imag ** 2)).sum(0)
    del z
    stream = torch.cuda.current_stream().cuda_stream
    fake = 1 << 20
    assert _static(1, NL, nb, nk + 1, fake, fake, nb, fake, 0) == -1  # one chunk row more than the maximum
    torch.cuda.synchronize()
    rc = _static(1, NL, nb, nk, zu.data_ptr(), occ.data_ptr(), nb, rho.data_ptr(), stream)
    assert rc == 0, _lib.lib().sgpu_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rho.fill_(float("nan"))
    rc = _static(1, NL, nb, nk, zu.data_ptr(), occ.data_ptr(), nb, rho.data_ptr(), stream)
    assert rc == 0, _lib.lib().sgpu_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    err = (rho - ref).abs().max().item() / ref.abs().max().item()
    assert err <= 1e-12, err
    del zu
    torch.cuda.empty_cache()
