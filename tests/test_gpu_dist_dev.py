"""The multi-GPU data plane on the device: the density and current written to
device buffers (sgpu_psi_rho_dev, sgpu_current_dev), all-reduced in place over
NCCL on the library's stream (dist.comm_summation_dev; a one-rank NCCL group,
since one GPU is available), and the potential rebuilt from the device density
(sgpu_update_vloc_dev), against the host path (sgpu_psi_rho, sgpu_current,
sgpu_update_vloc) and the CPU oracle.  Tolerance 1e-12 relative."""
import os
import socket

import numpy as np
import pytest

from _helpers import rel
from oracle import oracle as O
from salmon_b200 import dist as D, system as S

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_device_reductions_over_nccl(cuda_lib, precision):
    import datetime

    import torch
    import torch.distributed as dist
    from salmon_b200.rt import GpuSystem
    sysm, kAc, vpsl, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (2, 1, 1), 8, A=(0.0, 1e-2, 0.0))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        with GpuSystem(sysm, precision) as g:
            g.set_state(zu)
            g.set_vpsl(vpsl)
            g.set_vloc(vpsl)
            g.update_projector(kAc)
            g.hamiltonian(0.08, flag_current=True)
            z = g.get_state()
            rho = torch.empty(sysm.NL, dtype=torch.float64, device="cuda")
            jav = torch.empty(3, dtype=torch.float64, device="cuda")
            for _ in range(2):
                rho.fill_(float("nan"))
                jav.fill_(float("nan"))
                torch.cuda.synchronize()
                g.psi_rho_dev(rho.data_ptr())
                g.current_dev(kAc, jav.data_ptr())
                D.comm_summation_dev(g, rho)
                D.comm_summation_dev(g, jav)
                g.update_vloc_dev(rho.data_ptr())
                g.synchronize()
                torch.cuda.synchronize()
                assert rel(rho.cpu().numpy(), O.psi_rho(sysm, z)) < 1e-12
                assert rel(jav.cpu().numpy(), O.current(sysm, kAc, z)) < 1e-12
                v_dev = g.get_vloc()
            g.update_vloc(g.psi_rho_RT())   # the host path on the same density
            assert rel(v_dev, g.get_vloc()) < 1e-12
    finally:
        dist.destroy_process_group()
