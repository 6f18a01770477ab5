"""Bit-exact parity on the full benchmark workloads, every pair against the
oracle on all host threads (genomics/cpu/align_cpu.mojo:75-309 restated in
oracle/align_oracle.c):

  * 1,000,000 reads vs their 200 bp windows, band 32 (the headline workload);
  * 200,000 mixed-band pairs of 100-2,000 bp with N runs;
  * 100,000 long WFA pairs (100-10,000 bp, 1-10% divergence), exact-cover
    max_error, against the live-envelope oracle;
  * 24 of those pairs of 5-10 kbp against the statement-for-statement oracle
    (per-score reset of all 2*max_error+1 diagonals), each with its own
    exact-cover max_error;
  * the naive baselines (GB2_FLAG_NAIVE) on samples of the SW and WFA workloads.
"""
import os

import numpy as np
import pytest

from genomics_b200 import AlignConfig, SequenceBatch, WFAConfig, synth
from genomics_b200._lib import FLAG_NAIVE

pytestmark = pytest.mark.gpu

CFG0 = AlignConfig(2, -4, -4, -2, 32)
THREADS = os.cpu_count() or 1


def _sw_ref(O, q, r, cfg, bands=None):
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    return O.sw_batch(qp, qo, ql, rp, ro, rl, cfg.match_score, cfg.mismatch, cfg.gap_open,
                      cfg.gap_extend, cfg.band_width, bands=bands, threads=THREADS)


def _sw_mismatches(got, ref):
    sc, qe, re_ = ref
    return np.nonzero((got["score"] != sc) | (got["query_end"] != qe) | (got["ref_end"] != re_))[0]


def _subset(b, idx):
    p, m, o, l = b.arrays()
    return SequenceBatch.from_arrays(p, m, o[idx], l[idx])


def test_headline_workload_every_pair(device, oracle):
    q, r, _, _ = synth.generate(1, 1_000_000)
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    got = device.sw_banded(dq, dr, CFG0, batched=True)
    bad = _sw_mismatches(got, _sw_ref(oracle, q, r, CFG0))
    assert bad.size == 0, f"{bad.size} of 1,000,000 differ, first {bad[:5]}"
    dq.close()
    dr.close()


def test_mixed_band_workload_every_pair(device, oracle):
    q, r, bands, _ = synth.generate(3, 200_000)
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    ref = _sw_ref(oracle, q, r, CFG0, bands=bands)
    for batched in (True, False):
        got = device.sw_banded(dq, dr, CFG0, bands=bands, batched=batched)
        bad = _sw_mismatches(got, ref)
        assert bad.size == 0, f"batched={batched}: {bad.size} of 200,000 differ, first {bad[:5]}"
    # the naive baseline on a sample (it is slow by design)
    idx = np.arange(0, 200_000, 50)
    got = device.sw_banded(_subset(q, idx), _subset(r, idx), CFG0, bands=bands[idx],
                           batched=False, flags=FLAG_NAIVE)
    bad = _sw_mismatches(got, tuple(a[idx] for a in ref))
    assert bad.size == 0, f"naive: {bad.size} differ"
    dq.close()
    dr.close()


@pytest.fixture(scope="module")
def long_wfa():
    q, r, _, _ = synth.generate(2, 100_000)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    return q, r, WFAConfig(4, 6, 2, me)


def test_long_wfa_workload_every_pair(device, oracle, long_wfa):
    q, r, cfg = long_wfa
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    got = np.asarray(device.wfa_affine(dq, dr, cfg, batched=True))
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    want, _ = oracle.wfa_batch(qp, qo, ql, rp, ro, rl, 4, 6, 2, cfg.max_error, envelope=True,
                               threads=THREADS)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"{bad.size} of 100,000 differ, first {bad[:5]}"
    assert (got >= 0).all()
    # input order (plain) and the naive baseline on a sample
    assert (np.asarray(device.wfa_affine(dq, dr, cfg, batched=False)) == want).all()
    idx = np.arange(0, 100_000, 97)
    naive = np.asarray(device.wfa_affine(_subset(q, idx), _subset(r, idx), cfg, batched=False,
                                         flags=FLAG_NAIVE))
    assert (naive == want[idx]).all()
    dq.close()
    dr.close()


def test_long_pairs_against_statement_for_statement_oracle(device, oracle, long_wfa):
    """5-10 kbp pairs, each with its own exact-cover max_error, against the form of
    the oracle that resets all 2*max_error+1 diagonals per score as the reference
    does (align_cpu.mojo:153-156)."""
    q, r, _ = long_wfa
    ql, rl = q.lengths, r.lengths
    lmax = np.maximum(ql, rl)
    pick = np.nonzero((lmax >= 5000) & (lmax <= 10000))[0][:24]
    assert pick.size == 24
    qs, rs = _subset(q, pick), _subset(r, pick)
    qp, _, qo, qln = qs.arrays()
    rp, _, ro, rln = rs.arrays()
    for i in range(pick.size):
        me = int(4 * min(qln[i], rln[i]) + (6 + 2 * abs(int(qln[i]) - int(rln[i]))
                                            if qln[i] != rln[i] else 0))
        want, _ = oracle.wfa_batch(qp, qo[i:i + 1], qln[i:i + 1], rp, ro[i:i + 1],
                                   rln[i:i + 1], 4, 6, 2, me, envelope=False, threads=1)
        one_q = SequenceBatch.from_arrays(qp, np.zeros_like(qp), qo[i:i + 1], qln[i:i + 1])
        one_r = SequenceBatch.from_arrays(rp, np.zeros_like(rp), ro[i:i + 1], rln[i:i + 1])
        got = device.wfa_affine(one_q, one_r, WFAConfig(4, 6, 2, me))
        assert int(got[0]) == int(want[0]) and want[0] >= 0, (int(pick[i]), got[0], want[0])
