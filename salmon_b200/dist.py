"""k-point sharding over ranks (one process per GPU) and the per-step reductions.

The reference distributes k-points over the ranks of nproc_group_tdks
(control/initialization.f90:348-361) and sums the per-rank density and current
with comm_summation (common/psi_rho.f90:88, RT/current.f90:286); every rank
keeps the whole grid.  Here each rank holds one handle for its k-block; the
Taylor step has no exchange, and rho / J are reduced once per step over
torch.distributed (NCCL over NVLink on GPUs, gloo on CPU for the tests):
comm_summation for host values, comm_summation_dev for device buffers that
the library filled (sgpu_psi_rho_dev, sgpu_current_dev), reduced in place on
the library's stream with no host round trip.
"""
from __future__ import annotations

import copy

import numpy as np


def k_range(NK: int, world: int, rank: int):
    """1-based (NK_s, NK_e) of `rank`, the rule of initialization.f90:348-361:
    blocks of NK // world, the last NK % world ranks take one more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    ave, rem = NK // world, NK % world
    if rem == 0 or rank < (world - 1) - rem + 1:
        return ave * rank + 1, ave * (rank + 1)
    return NK - (ave + 1) * ((world - 1) - rank) - ave, NK - (ave + 1) * ((world - 1) - rank)


def local_system(sysm, rank: int, world: int):
    """A copy of the system description restricted to the rank's k-block."""
    s = copy.copy(sysm)
    s.NK_s, s.NK_e = k_range(sysm.NK, world, rank)
    if s.NK_e < s.NK_s:
        raise ValueError(f"rank {rank} has no k-points (NK={sysm.NK}, world={world})")
    return s


def local_orbitals(zu_all, sysm_local):
    """The rank's block of zu(NL, NB, NK) (C-order (NK, NB, NL) numpy array)."""
    return np.ascontiguousarray(zu_all[sysm_local.NK_s - 1:sysm_local.NK_e])


def comm_summation(x, group=None):
    """Allreduce-sum of a numpy array (or float) over the default process group;
    on NCCL the values travel through the current CUDA device."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    arr = np.asarray(x, dtype=np.float64)
    t = torch.from_numpy(np.ascontiguousarray(arr).copy())
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    return out if np.ndim(x) else float(out)


def comm_summation_dev(g, t, group=None):
    """In-place allreduce-sum of the CUDA tensor t over the default process group,
    ordered on the stream of the GpuSystem g: after the kernels that filled t
    (sgpu_psi_rho_dev / sgpu_current_dev on g.stream) and before the handle's
    next work (e.g. sgpu_update_vloc_dev reading t).  No host copy."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return t
    with torch.cuda.stream(torch.cuda.ExternalStream(g.stream)):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def local_descriptors_valid(sysm, world: int):
    """Every rank's k-block descriptor passes the library's host-side checks
    (sgpu_check_desc; no device needed).  Returns the (NK_s, NK_e) blocks."""
    from .rt import check_desc
    blocks = []
    for r in range(world):
        loc = local_system(sysm, r, world)
        check_desc(loc)
        blocks.append((loc.NK_s, loc.NK_e))
    return blocks
