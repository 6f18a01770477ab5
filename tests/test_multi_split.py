"""One pair list over several devices, host side (no GPU): the work-unit
partitioner of the C ABI (gb2_partition_pairs) and, with two gloo ranks on the
CPU, the partition -> per-rank slice -> all_gather path of genomics_b200.multi.
On the CPU the oracle stands in for each rank's device, so what is tested is
the split and the gather: the gathered results must equal one oracle pass over
the whole list, in input order."""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT


def _work(ql, rl, bands, kind):
    if kind == 0:
        return ql * (2 * bands.astype(np.int64) + 1) + 1024
    l = np.maximum(ql, rl).astype(np.float64)
    return l * l + 1024


@pytest.mark.parametrize("kind,wl", [(0, 3), (1, 2)])
@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_splits_by_work(kind, wl, parts):
    from genomics_b200 import multi, synth
    q, r, bands, _ = synth.generate(wl, 5000)
    ql, rl = q.lengths, r.lengths
    b = multi.partition(ql, rl, parts, kind, 32, bands if kind == 0 else None)
    assert b[0] == 0 and b[-1] == 5000 and (np.diff(b) >= 0).all()
    w = _work(ql, rl, bands if kind == 0 else np.full(5000, 32), kind)
    share = np.add.reduceat(w, b[:-1]) if parts > 1 else np.array([w.sum()])
    share = np.array([w[b[k]:b[k + 1]].sum() for k in range(parts)])
    # every part is within one pair's work of the ideal share
    assert (np.abs(share - w.sum() / parts) <= w.max() + 1).all()


def test_partition_edges():
    from genomics_b200 import _lib, multi
    assert list(multi.partition([], [], 3)) == [0, 0, 0, 0]
    b = multi.partition([10, 10_000, 10], [10, 10_000, 10], 4, kind=1)
    assert b[0] == 0 and b[-1] == 3 and (np.diff(b) >= 0).all()
    L = _lib.lib()
    out = np.zeros(3, np.int64)
    ql = np.array([5, -1], np.int64)
    p = lambda a: a.ctypes.data
    assert L.gb2_partition_pairs(p(ql), p(ql), None, 8, 0, 2, 2, p(out)) == _lib.GB2_EINVAL
    assert L.gb2_partition_pairs(p(ql), p(ql), None, 8, 2, 1, 2, p(out)) == _lib.GB2_EINVAL
    assert L.gb2_partition_pairs(p(ql), p(ql), None, 8, 0, 1, 0, p(out)) == _lib.GB2_EINVAL


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_slice(O, q, r, i0, i1, kind, bands):
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    sl = slice(i0, i1)
    if kind == 0:
        sc, qe, re_ = O.sw_batch(qp, qo[sl], ql[sl], rp, ro[sl], rl[sl], 2, -4, -4, -2, 32,
                                 bands=bands[sl], threads=2)
        return np.stack([sc, qe, re_], axis=1).astype(np.int32)
    me = 4 * int(np.minimum(ql, rl).max()) + 6 + 2 * int(np.abs(ql - rl).max())
    cost, _ = O.wfa_batch(qp, qo[sl], ql[sl], rp, ro[sl], rl[sl], 4, 6, 2, me, threads=2)
    return cost.reshape(-1, 1).astype(np.int32)


def _worker(rank, world, port, out_q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    for p in (os.path.join(ROOT, "computational-genomics-mojo_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import datetime

    import oracle as O
    import torch.distributed as dist
    from genomics_b200 import multi, synth
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    res = {}
    for kind, wl in ((0, 3), (1, 2)):
        q, r, bands, _ = synth.generate(wl, 1500)
        bounds = multi.partition(q.lengths, r.lengths, world, kind, 32,
                                 bands if kind == 0 else None)
        local = _oracle_slice(O, q, r, int(bounds[rank]), int(bounds[rank + 1]), kind, bands)
        full = multi.gather_slices(local, bounds)
        res[kind] = (full, bounds)
    out_q.put((rank, res))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_partition_and_gather_gloo(oracle):
    import torch.multiprocessing as mp
    from genomics_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for kind, wl in ((0, 3), (1, 2)):
        qb, rb, bands, _ = synth.generate(wl, 1500)
        want = _oracle_slice(oracle, qb, rb, 0, 1500, kind, bands)
        for rank in (0, 1):
            full, bounds = got[rank][kind]
            assert 0 < bounds[1] < 1500  # both ranks had pairs
            assert (full == want).all(), (kind, rank)
