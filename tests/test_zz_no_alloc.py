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
