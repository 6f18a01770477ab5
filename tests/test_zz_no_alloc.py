"""gb2_wfa_affine_noalloc: the WFA entry point for callers that cannot call
cudaMalloc (their device memory belongs to a host runtime's allocator, or
they live inside a fixed memory budget).  It must give exactly the costs of
the allocating entry point, call after call, using only the caller's buffers
and the library's fixed scratch array.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from genomics_b200 import WFAConfig, _lib, synth

pytestmark = pytest.mark.gpu


def _device_copies(torch, batch):
    """Device copies of a SequenceBatch, allocated by the test (torch)."""
    p, _, o, l = batch.arrays()
    return (torch.from_numpy(p.view(np.int64).copy()).cuda(),
            torch.from_numpy(o.copy()).cuda(), torch.from_numpy(l.copy()).cuda())


def test_noalloc_matches_allocating_entry_point(device):
    torch = pytest.importorskip("torch")
    q, r, _, _ = synth.generate(2, 300, seed=2024)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    cfg = WFAConfig(4, 6, 2, me)
    want = device.wfa_affine(q, r, cfg)  # the existing, allocating entry point
    assert (want >= 0).all()

    qp, qo, ql = _device_copies(torch, q)
    rp, ro, rl = _device_copies(torch, r)
    n = int(ql.numel())
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    c = _lib.WfaCfg(4, 6, 2, me)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    for call in range(2):  # two calls in a row share (and reuse) the fixed scratch
        out.fill_(-7)
        rc = L.gb2_wfa_affine_noalloc(
            ctypes.c_void_p(qp.data_ptr()), qp.numel(), ctypes.c_void_p(qo.data_ptr()),
            ctypes.c_void_p(ql.data_ptr()), ctypes.c_void_p(rp.data_ptr()), rp.numel(),
            ctypes.c_void_p(ro.data_ptr()), ctypes.c_void_p(rl.data_ptr()),
            int(q.lengths.max()), int(r.lengths.max()), ctypes.byref(c), n,
            ctypes.c_void_p(out.data_ptr()), stream)
        assert rc == _lib.GB2_OK, (call, rc)
        got = out.cpu().numpy()
        assert (got == want).all(), (call, np.nonzero(got != want)[0][:5])


def test_noalloc_rejects_sizes_beyond_its_scratch(device):
    torch = pytest.importorskip("torch")
    q, r, _, _ = synth.generate(2, 4, seed=1)
    qp, qo, ql = _device_copies(torch, q)
    rp, ro, rl = _device_copies(torch, r)
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    c = _lib.WfaCfg(4, 6, 2, 1000)
    L = _lib.lib()
    args = lambda mq, mr: (ctypes.c_void_p(qp.data_ptr()), qp.numel(),
                           ctypes.c_void_p(qo.data_ptr()), ctypes.c_void_p(ql.data_ptr()),
                           ctypes.c_void_p(rp.data_ptr()), rp.numel(),
                           ctypes.c_void_p(ro.data_ptr()), ctypes.c_void_p(rl.data_ptr()),
                           mq, mr, ctypes.byref(c), 4, ctypes.c_void_p(out.data_ptr()), None)
    # rings for 4 warps of 9 x 600k int32 each exceed the 32 MiB scratch
    assert L.gb2_wfa_affine_noalloc(*args(300_000, 300_000)) == _lib.GB2_ESCRATCH
    assert L.gb2_strerror(_lib.GB2_ESCRATCH) == b"request exceeds the fixed no-allocation scratch"


def test_noalloc_flags_pairs_longer_than_declared(device):
    """A pair longer than the stated bounds gets cost -2 and the call returns
    GB2_EINVAL; the next call with the right bounds is clean (the shared header
    was cleared) and equals the allocating entry point."""
    torch = pytest.importorskip("torch")
    import random
    rng = random.Random(11)
    rand = lambda n: "".join(rng.choice("ACGT") for _ in range(n))
    qs = [rand(rng.randint(150, 240)) for _ in range(8)] + [rand(2000)]
    rs = [s[:50] + "T" + s[51:] for s in qs]
    from genomics_b200 import SequenceBatch
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    cfg = WFAConfig(4, 6, 2, 4000)
    want = device.wfa_affine(q, r, cfg)
    qp, qo, ql = _device_copies(torch, q)
    rp, ro, rl = _device_copies(torch, r)
    n = len(qs)
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    c = _lib.WfaCfg(4, 6, 2, 4000)
    L = _lib.lib()

    def call(mq, mr):
        out.fill_(-7)
        rc = L.gb2_wfa_affine_noalloc(
            ctypes.c_void_p(qp.data_ptr()), qp.numel(), ctypes.c_void_p(qo.data_ptr()),
            ctypes.c_void_p(ql.data_ptr()), ctypes.c_void_p(rp.data_ptr()), rp.numel(),
            ctypes.c_void_p(ro.data_ptr()), ctypes.c_void_p(rl.data_ptr()), mq, mr,
            ctypes.byref(c), n, ctypes.c_void_p(out.data_ptr()), None)
        torch.cuda.synchronize()
        return rc, out.cpu().numpy()

    rc, got = call(250, 250)  # the last pair is 2,000 bases: longer than declared
    assert rc == _lib.GB2_EINVAL
    assert got[-1] == -2
    assert (got[:-1] == want[:-1]).all()
    rc, got = call(int(q.lengths.max()), int(r.lengths.max()))
    assert rc == _lib.GB2_OK
    assert (got == want).all()
