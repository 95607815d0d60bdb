"""k-point sharding host logic with world_size 2 over gloo on CPU: each rank
builds its k-block's descriptor and has the library check it on the host
(sgpu_check_desc, no device), computes rho, J and the energy terms of its block
with the CPU oracle, and the sums over ranks equal the single-process results
(1e-12)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from salmon_b200 import dist as D


def test_k_range_matches_the_reference_rule():
    for NK in (1, 3, 7, 8, 64, 65):
        for world in range(1, min(NK, 9) + 1):
            blocks = [D.k_range(NK, world, r) for r in range(world)]
            covered = [k for s, e in blocks for k in range(s, e + 1)]
            assert covered == list(range(1, NK + 1))
            sizes = [e - s + 1 for s, e in blocks]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from salmon_b200 import system as S
        from salmon_b200.rt import SalmonGPUError, check_desc
        sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=3, nb=4)
        loc = D.local_system(sysm, rank, world)
        # the library's host-side checks of this rank's descriptor (no device call)
        check_desc(loc)
        d = loc.desc()
        assert (d.NK, d.NK_s, d.NK_e) == (sysm.NK,) + D.k_range(sysm.NK, world, rank)
        bad = D.local_system(sysm, rank, world)
        bad.NK_e = sysm.NK + 1
        try:
            check_desc(bad)
            raise AssertionError("a k range beyond NK was accepted")
        except SalmonGPUError:
            pass
        zl = D.local_orbitals(zu, loc)
        rho = D.comm_summation(O.psi_rho(loc, zl))
        jav = D.comm_summation(O.current(loc, kAc, zl))
        ek, en = O.energy_terms(loc, kAc, zl)
        ek, en = D.comm_summation(ek), D.comm_summation(en)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), rho=rho, jav=jav, e=np.array([ek, en]),
                 ks=np.array([loc.NK_s, loc.NK_e]))
    finally:
        dist.destroy_process_group()


def test_sharded_reductions_equal_single_process(tmp_path):
    from oracle import oracle as O
    from salmon_b200 import system as S
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    sysm, kAc, vloc, zu = S.small_system(8, 8, 10, nk=3, nb=4)
    rho0, j0 = O.psi_rho(sysm, zu), O.current(sysm, kAc, zu)
    e0 = np.array(O.energy_terms(sysm, kAc, zu))
    res = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    assert [tuple(r["ks"]) for r in res] == [(1, 1), (2, 3)]
    for r in res:
        np.testing.assert_allclose(r["rho"], rho0, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(r["jav"], j0, rtol=1e-12, atol=1e-16)
        np.testing.assert_allclose(r["e"], e0, rtol=1e-12)


def test_every_rank_descriptor_passes_the_library_checks():
    from salmon_b200 import system as S
    sysm, kAc, vloc, zu = S.microbench_system(16, nkgrid=(4, 4, 4), Nb=8, with_orbitals=False)
    for world in (1, 2, 3, 8):
        blocks = D.local_descriptors_valid(sysm, world)
        assert blocks == [D.k_range(sysm.NK, world, r) for r in range(world)]
