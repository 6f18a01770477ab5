"""Failure handling on the host: injected allocation failures, a server wait
that runs out, cancellation of queued requests and malformed requests.

None of these faults a GPU: allocations fail through the library's own
countdown hook before any CUDA call is made, waits run out on the host, and
bad requests are rejected at submit.  After each failure the context must
answer the next call correctly.  (The reference's only failure report is
WFA's -1 past max_error, genomics/cpu/align_cpu.mojo:226.)
"""
import ctypes

import numpy as np
import pytest

from genomics_b200 import AlignConfig, GenomicsDevice, SequenceBatch, WFAConfig, _lib, synth
from genomics_b200._lib import GenomicsError
from genomics_b200.serve import SW, WFA, AlignmentServer

pytestmark = pytest.mark.gpu

SWC = AlignConfig(2, -4, -4, -2, 32)


def _arm(kind, nth):
    assert _lib.lib().gb2_debug_fail_alloc(kind, nth) == _lib.GB2_OK


def test_injected_device_allocation_failures():
    """The nth device allocation of a call fails: the call returns GB2_ENOMEM, and
    the same context then gives the right results (fresh context, so the call
    itself allocates its buffers)."""
    q, r, bands, _ = synth.generate(3, 600)
    qw, rw, _, _ = synth.generate(2, 300)
    cfg = WFAConfig(4, 6, 2, synth.wfa_max_error_cover(qw, rw, 4, 6, 2))
    ref_dev = GenomicsDevice(0)
    try:
        want_sw = ref_dev.sw_banded(q, r, SWC, bands=bands)
        want_wfa = ref_dev.wfa_affine(qw, rw, cfg)
    finally:
        ref_dev.close()
    failures = 0
    for nth in range(6):
        dev = GenomicsDevice(0)
        try:
            dq, dr = dev.upload_batch(q), dev.upload_batch(r)
            dqw, drw = dev.upload_batch(qw), dev.upload_batch(rw)
            for name, run, want in (
                    ("sw", lambda: dev.sw_banded(dq, dr, SWC, bands=bands), want_sw),
                    ("wfa", lambda: dev.wfa_affine(dqw, drw, cfg), want_wfa)):
                _arm(_lib.GB2_ALLOC_DEVICE, nth)
                try:
                    got = run()
                    # fewer than nth + 1 allocations: the call ran normally
                    assert (np.asarray(got) == np.asarray(want)).all(), (name, nth)
                except GenomicsError as e:
                    assert e.code == _lib.GB2_ENOMEM, (name, nth, e)
                    failures += 1
                finally:
                    _arm(_lib.GB2_ALLOC_DEVICE, -1)
                assert (np.asarray(run()) == np.asarray(want)).all(), (name, nth, "after")
            dev.synchronize()
        finally:
            _arm(_lib.GB2_ALLOC_DEVICE, -1)
            dev.close()
    assert failures >= 6  # at least the first allocations of both calls failed


def test_injected_pinned_allocation_failure():
    """A pinned staging allocation of the end-to-end path fails: GB2_ENOMEM,
    then the same call succeeds."""
    q, r, _, _ = synth.generate(1, 20000)
    dev = GenomicsDevice(0)
    failures = 0
    try:
        want = None
        for nth in range(3):
            _arm(_lib.GB2_ALLOC_PINNED, nth)
            try:
                got = dev.sw_banded(q, r, SWC, flags=_lib.FLAG_BATCHED)
                if want is not None:
                    assert (got == want).all()
            except GenomicsError as e:
                assert e.code == _lib.GB2_ENOMEM, e
                failures += 1
            finally:
                _arm(_lib.GB2_ALLOC_PINNED, -1)
            again = dev.sw_banded(q, r, SWC)
            if want is None:
                want = again
            assert (again == want).all()
        assert failures >= 1  # the first call's staging allocation failed
    finally:
        _arm(_lib.GB2_ALLOC_PINNED, -1)
        dev.close()


def _req(n=40, seed=9):
    q, r, bands, kinds = synth.generate(4, n, seed=seed)
    keep = np.nonzero((q.lengths <= 2000) & (r.lengths <= 2000))[0]
    p, _, o, l = q.arrays()
    pr, _, orr, lr = r.arrays()
    qs = SequenceBatch.from_arrays(p, np.zeros_like(p), o[keep], l[keep])
    rs = SequenceBatch.from_arrays(pr, np.zeros_like(pr), orr[keep], lr[keep])
    return qs, rs, bands[keep], kinds[keep]


def _expected(dev, req, wcfg):
    q, r, bands, kinds = req
    sw = dev.sw_banded(q, r, SWC, bands=bands)
    wfa = dev.wfa_affine(q, r, wcfg)
    return sw, wfa


def _same(res, exp, kinds):
    sw, wfa = res
    esw, ewfa = exp
    s = kinds == SW
    assert (sw[s] == esw[s]).all()
    assert (wfa[~s] == ewfa[~s]).all()


def test_server_wait_times_out_then_completes(device):
    wcfg = WFAConfig(4, 6, 2, 20000)
    req = _req()
    exp = _expected(device, req, wcfg)
    with AlignmentServer(device, hbm_budget_bytes=4 << 30, max_inflight_groups=2) as srv:
        srv.hold(True)
        q, r, bands, kinds = req
        pr = srv.submit(q, r, SWC, wcfg, kinds=kinds, bands=bands)
        with pytest.raises(TimeoutError):
            pr.wait(50)  # admission is held: the wait runs out (GB2_ETIMEOUT)
        assert not pr.done()
        srv.hold(False)
        _same(pr.wait(600_000), exp, kinds)


def test_server_cancels_queued_requests(device):
    wcfg = WFAConfig(4, 6, 2, 20000)
    reqs = [_req(40, seed=s) for s in (1, 2, 3)]
    exps = [_expected(device, rq, wcfg) for rq in reqs]
    with AlignmentServer(device, hbm_budget_bytes=4 << 30, max_inflight_groups=2) as srv:
        srv.hold(True)
        prs = [srv.submit(q, r, SWC, wcfg, kinds=k, bands=b) for q, r, b, k in reqs]
        prs[1].cancel()
        with pytest.raises(GenomicsError) as ei:
            prs[1].cancel()  # no longer queued
        assert ei.value.code == _lib.GB2_ESTATE
        srv.hold(False)
        for i in (0, 2):
            _same(prs[i].wait(600_000), exps[i], reqs[i][3])
        with pytest.raises(GenomicsError) as ei:
            prs[1].wait(600_000)
        assert ei.value.code == _lib.GB2_ECANCELED
        # done requests cannot be cancelled; unknown tickets are invalid
        L = _lib.lib()
        done = srv.submit(*reqs[0][:2], SWC, wcfg, kinds=reqs[0][3], bands=reqs[0][2])
        done.wait(600_000)
        assert L.gb2_server_cancel(srv.handle, 987654321) == _lib.GB2_EINVAL
        st = srv.stats()
        assert st["cancelled"] == 1 and st["failed"] == 0


def test_server_rejects_malformed_requests(device):
    wcfg = WFAConfig(4, 6, 2, 2000)
    q, r, bands, kinds = _req(40)
    kinds = np.ascontiguousarray(kinds, np.int32)
    bands = np.ascontiguousarray(bands, np.int32)
    n = kinds.size
    assert n >= 4
    L = _lib.lib()
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    sw_out = np.zeros(n * 3, np.int32)
    wfa_out = np.zeros(n, np.int32)
    P = lambda a: ctypes.c_void_p(a.ctypes.data) if a is not None else None
    from genomics_b200.device import _sw_cfg, _wfa_cfg

    def submit(qo_=qo, ql_=ql, kinds_=kinds, bands_=bands, sw=sw_out, wfa=wfa_out, nn=n):
        req = _lib.Request(nn, P(qp), P(qo_), P(ql_), P(rp), P(ro), P(rl), P(kinds_),
                           P(bands_), _sw_cfg(SWC), _wfa_cfg(wcfg), P(sw), P(wfa))
        t = ctypes.c_uint64()
        return L.gb2_server_submit(srv.handle, ctypes.byref(req), ctypes.byref(t))

    with AlignmentServer(device, hbm_budget_bytes=4 << 30) as srv:
        before = srv.stats()["submitted"]
        neg_len = ql.copy(); neg_len[3] = -5
        neg_off = qo.copy(); neg_off[2] = -1
        bad_kind = kinds.astype(np.int32).copy(); bad_kind[1] = 2
        neg_band = bands.astype(np.int32).copy(); neg_band[0] = -3
        all_sw = np.zeros(n, np.int32)
        all_wfa = np.ones(n, np.int32)
        huge = ql.copy(); huge[0] = 1 << 31
        assert submit(ql_=neg_len) == _lib.GB2_EINVAL
        assert submit(qo_=neg_off) == _lib.GB2_EINVAL
        assert submit(kinds_=bad_kind) == _lib.GB2_EINVAL
        assert submit(kinds_=all_sw, bands_=neg_band) == _lib.GB2_EINVAL
        assert submit(kinds_=all_sw, sw=None) == _lib.GB2_EINVAL
        assert submit(kinds_=all_wfa, wfa=None) == _lib.GB2_EINVAL
        assert submit(kinds_=all_wfa, ql_=huge) == _lib.GB2_ERANGE
        assert submit(nn=-1) == _lib.GB2_EINVAL
        assert srv.stats()["submitted"] == before  # nothing was queued
        assert submit() == _lib.GB2_OK  # the well-formed request still goes through
