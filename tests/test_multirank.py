"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): ranks meet at
barriers, the step time is the max over ranks, work units add up, and every
rank aligns its own seeded shard (weak scaling, no collective on the data)."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "computational-genomics-mojo_b200"))
    import bench
    from genomics_b200 import synth
    d = bench.Dist()
    d.barrier()
    t = d.max(10.0 + rank)          # slowest rank decides the step time
    units = d.sum(100.0 * (rank + 1))
    seed = synth.default_seed(1) + 7919 * rank
    qb, _, _, _ = synth.generate(0, 16, seed=seed)
    q.put((rank, t, units, seed, int(qb.packed.sum() % (1 << 62))))
    d.barrier()
    d.close()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [11.0, 11.0]
    assert [o[2] for o in out] == [300.0, 300.0]
    assert out[0][3] != out[1][3] and out[0][4] != out[1][4]  # distinct shards
