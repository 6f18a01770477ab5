"""Serving layer (gb2_server_*): every request's results equal the oracle and
are the same whether the request runs alone or mixed with others in flight."""
import threading

import numpy as np
import pytest

from genomics_b200 import AlignConfig, SequenceBatch, WFAConfig, synth
from genomics_b200._lib import GenomicsError
from genomics_b200.serve import SW, WFA, AlignmentServer

pytestmark = pytest.mark.gpu

SWC = AlignConfig(2, -4, -4, -2, 32)


def _subset(batch, idx):
    p, m, o, l = batch.arrays()
    parts, offs, lens, w = [], [], [], 0
    for i in idx:
        nw = (int(l[i]) + 31) // 32
        parts.append(p[o[i]:o[i] + nw])
        offs.append(w)
        lens.append(int(l[i]))
        w += nw
    cat = np.concatenate(parts) if parts else np.zeros(0, np.uint64)
    return SequenceBatch.from_arrays(cat, np.zeros_like(cat), np.array(offs, np.int64),
                                     np.array(lens, np.int64))


@pytest.fixture(scope="module")
def pool():
    """Serving-mix pairs (SW band 32/64/128 or WFA) no longer than 3,000 bp."""
    q, r, bands, kinds = synth.generate(4, 6000, seed=404)
    keep = np.nonzero((q.lengths <= 3000) & (r.lengths <= 3000))[0][:1500]
    return _subset(q, keep), _subset(r, keep), bands[keep], kinds[keep]


def _requests(pool, sizes, rng):
    q, r, bands, kinds = pool
    n = q.count
    out, start = [], 0
    for s in sizes:
        idx = (np.arange(s) + start) % n
        start += s
        out.append((_subset(q, idx), _subset(r, idx), bands[idx], kinds[idx]))
    return out


def _expected(oracle, req, wcfg):
    q, r, bands, kinds = req
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    sc, qe, re_ = oracle.sw_batch(qp, qo, ql, rp, ro, rl, 2, -4, -4, -2, 32, bands=bands)
    cost, _ = oracle.wfa_batch(qp, qo, ql, rp, ro, rl, wcfg.x, wcfg.o, wcfg.e, wcfg.max_error)
    return sc, qe, re_, cost


def _check(res, exp, kinds, what):
    sw, wfa = res
    sc, qe, re_, cost = exp
    s = kinds == SW
    assert (sw["score"][s] == sc[s]).all(), what
    assert (sw["query_end"][s] == qe[s]).all() and (sw["ref_end"][s] == re_[s]).all(), what
    assert (wfa[~s] == cost[~s]).all(), what


def test_alone_and_in_the_mix(device, oracle, pool):
    wcfg = WFAConfig(4, 6, 2, 30000)
    rng = np.random.default_rng(5)
    reqs = _requests(pool, [1, 7, 64, 300, 33, 512, 2, 128, 900, 5], rng)
    exps = [_expected(oracle, rq, wcfg) for rq in reqs]
    with AlignmentServer(device, hbm_budget_bytes=4 << 30, max_inflight_groups=4) as srv:
        # each request alone
        alone = []
        for rq, ex in zip(reqs, exps):
            pr = srv.submit(rq[0], rq[1], SWC, wcfg, kinds=rq[3], bands=rq[2])
            res = pr.wait(120_000)
            _check(res, ex, rq[3], "alone")
            alone.append((res[0].copy(), res[1].copy()))
        # all of them at once from several threads, twice over
        results = {}

        def client(k):
            mine = []
            for j in range(k, len(reqs), 3):
                rq = reqs[j]
                mine.append((j, srv.submit(rq[0], rq[1], SWC, wcfg, kinds=rq[3], bands=rq[2])))
            for j, pr in mine:
                results.setdefault(j, []).append(pr.wait(120_000))

        for _round in range(2):
            th = [threading.Thread(target=client, args=(k,)) for k in range(3)]
            for t in th:
                t.start()
            for t in th:
                t.join()
        for j, rq in enumerate(reqs):
            for res in results[j]:
                _check(res, exps[j], rq[3], f"mixed request {j}")
                s = rq[3] == SW
                assert (res[0][s] == alone[j][0][s]).all() and (res[1][~s] == alone[j][1][~s]).all()
        st = srv.stats()
        assert st["completed"] == 3 * len(reqs) and st["failed"] == 0
        assert st["groups_launched"] >= 1


def test_tight_budget_queues_but_completes(device, oracle, pool):
    wcfg = WFAConfig(4, 6, 2, 30000)
    reqs = _requests(pool, [200] * 8, np.random.default_rng(1))
    budget = 200 << 20
    with AlignmentServer(device, hbm_budget_bytes=budget, max_inflight_groups=2,
                         max_group_pairs=400) as srv:
        prs = [srv.submit(rq[0], rq[1], SWC, wcfg, kinds=rq[3], bands=rq[2]) for rq in reqs]
        for rq, pr in zip(reqs, prs):
            _check(pr.wait(120_000), _expected(oracle, rq, wcfg), rq[3], "tight budget")
            assert pr.latency_ms is not None and pr.latency_ms >= 0
        st = srv.stats()
        assert st["peak_inflight_bytes"] <= budget
        assert st["groups_launched"] >= 2


def test_request_larger_than_budget_is_rejected(device, pool):
    q, r, bands, kinds = pool
    with AlignmentServer(device, hbm_budget_bytes=1 << 20, max_inflight_groups=1) as srv:
        with pytest.raises(GenomicsError):
            srv.submit(q, r, SWC, WFAConfig(4, 6, 2, 30000), kinds=kinds, bands=bands)


def test_empty_request(device):
    e = SequenceBatch.from_strings([])
    with AlignmentServer(device) as srv:
        sw, wfa = srv.submit(e, e, SWC, WFAConfig(4, 6, 2, 10)).wait(10_000)
        assert sw.size == 0 and wfa.size == 0


def test_long_wfa_pairs_alone_and_in_the_mix(device, oracle):
    """Requests holding 8-20 kbp WFA pairs at up to 15% divergence (the pairs that
    climb to the largest WFA tiers and to int32 rings) give the same costs alone
    and mixed with short requests in flight, and equal the oracle."""
    q, r, bands, kinds = synth.generate(4, 4000, seed=808)
    lmax = np.maximum(q.lengths, r.lengths)
    longs = np.nonzero((kinds == WFA) & (lmax >= 8000))[0][:6]
    shorts = np.nonzero(lmax <= 1500)[0][:400]
    assert longs.size == 6
    wcfg = WFAConfig(4, 6, 2, synth.wfa_max_error_cover(q, r, 4, 6, 2))
    big = (_subset(q, longs), _subset(r, longs), bands[longs], kinds[longs])
    exp_big = _expected(oracle, big, wcfg)
    small = [(_subset(q, shorts[i::4]), _subset(r, shorts[i::4]), bands[shorts[i::4]],
              kinds[shorts[i::4]]) for i in range(4)]
    with AlignmentServer(device, hbm_budget_bytes=16 << 30, max_inflight_groups=4) as srv:
        alone = srv.submit(big[0], big[1], SWC, wcfg, kinds=big[3], bands=big[2]).wait(600_000)
        _check(alone, exp_big, big[3], "long pairs alone")
        prs = [srv.submit(s[0], s[1], SWC, wcfg, kinds=s[3], bands=s[2]) for s in small[:2]]
        pb = srv.submit(big[0], big[1], SWC, wcfg, kinds=big[3], bands=big[2])
        prs += [srv.submit(s[0], s[1], SWC, wcfg, kinds=s[3], bands=s[2]) for s in small[2:]]
        mixed = pb.wait(600_000)
        assert (mixed[1] == alone[1]).all()
        _check(mixed, exp_big, big[3], "long pairs in the mix")
        for s, pr in zip(small, prs):
            _check(pr.wait(600_000), _expected(oracle, s, wcfg), s[3], "short requests")
