"""Multi-rank host logic on CPU: two gloo ranks shard an ensemble of Arnoldi problems.

The problems run on the CPU oracle (oracle/arnoldi.py) in place of the GPU; the test checks
the split, the gather order, that each sharded problem equals its single-process run bit for
bit, and the max-over-ranks clock.
"""
import os
import socket

import numpy as np
import pytest

from gatt_dns_b200.shard import member_range


def test_member_range_covers_once():
    for total in range(0, 11):
        for world in range(1, 5):
            got = []
            for r in range(world):
                lo, hi = member_range(total, world, r)
                got.extend(range(lo, hi))
            assert got == list(range(total))


def _problem_setup():
    from gatt_dns_b200 import case as cs
    c = cs.periodic_box(n=12)
    base = cs.solenoidal_turbulence(c, seed=1234)
    rng = np.random.default_rng(5)
    v0 = []
    for _ in range(3):
        d = {k: np.zeros((12, 12, 12), order="F") for k in "UVWRE"}
        d["U"][...] = rng.standard_normal((12, 12, 12))
        d["V"][...] = rng.standard_normal((12, 12, 12))
        v0.append(d)
    return c, base, v0


def _runner(c, base):
    from oracle import Oracle
    from oracle.arnoldi import arnoldi
    o = Oracle(c, threads=1)
    return lambda vs: np.stack([arnoldi(o, c, base, v, 2, 2, 0.01, 1e-4) for v in vs])


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from gatt_dns_b200.shard import arnoldi_sharded, max_over_ranks
    c, base, v0 = _problem_setup()
    H = arnoldi_sharded(_runner(c, base), v0, dist=dist)
    t = max_over_ranks(1.0 + rank, dist=dist)
    np.save(os.path.join(out, "H%d.npy" % rank), H)
    np.save(os.path.join(out, "t%d.npy" % rank), np.array([t]))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_shard_arnoldi(tmp_path, oracle_lib):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    c, base, v0 = _problem_setup()
    ref = _runner(c, base)(v0)
    for r in range(world):
        H = np.load(tmp_path / ("H%d.npy" % r))
        assert H.shape == ref.shape
        assert np.array_equal(H, ref)
        assert float(np.load(tmp_path / ("t%d.npy" % r))[0]) == 2.0
