"""Gap-affine WFA on the GPU against the oracle: bit-exact costs (-1 past
max_error), through the C ABI."""
import random

import numpy as np
import pytest

import genomics_b200 as G
from genomics_b200 import SequenceBatch, WFAConfig, synth
from genomics_b200._lib import GenomicsError

pytestmark = pytest.mark.gpu


def oracle_wfa(O, q, r, cfg, envelope=True):
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    out, _ = O.wfa_batch(qp, qo, ql, rp, ro, rl, cfg.x, cfg.o, cfg.e, cfg.max_error,
                         envelope=envelope)
    return out


def assert_same(got, ref, what=""):
    bad = np.nonzero(got != ref)[0]
    assert bad.size == 0, f"{what}: {bad.size} mismatches, first {bad[:5]} got {got[bad[:5]]} want {ref[bad[:5]]}"


def test_known_answers_dropin(device, known):
    cfg = G.default_wfa_config()
    for case in known["wfa"]:
        qb = SequenceBatch.from_strings([case["q"]])
        rb = SequenceBatch.from_strings([case["r"]])
        assert G.wfa_affine_cpu(G.get_view(qb, 0), G.get_view(rb, 0), cfg) == case["cost"], case["src"]


def _mutated_pairs(rng, n, maxlen):
    qs, rs = [], []
    for _ in range(n):
        q = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, maxlen)))
        if rng.random() < 0.8:
            r = list(q)
            for _k in range(rng.randint(0, max(1, len(q) // 10))):
                pos = rng.randint(0, max(len(r) - 1, 0))
                op = rng.random()
                if op < 0.6 and r:
                    r[pos] = rng.choice("ACGT")
                elif op < 0.8:
                    r[pos:pos] = rng.choice("ACGT") * rng.randint(1, 4)
                elif r:
                    del r[pos:pos + rng.randint(1, 4)]
            r = "".join(r)
        else:
            r = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, maxlen)))
        qs.append(q)
        rs.append(r)
    return SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)


@pytest.mark.parametrize("pen", [(4, 6, 2), (2, 3, 1), (1, 0, 1), (6, 4, 2), (3, 5, 2), (5, 2, 3)])
def test_random_pairs(device, oracle, pen):
    rng = random.Random(sum(pen))
    q, r = _mutated_pairs(rng, 400, 400)
    for me in (0, 7, 60, 200, 4000):
        cfg = WFAConfig(*pen, me)
        ref = oracle_wfa(oracle, q, r, cfg)
        for batched in (True, False):
            assert_same(device.wfa_affine(q, r, cfg, batched=batched), ref, f"{pen} me={me}")


def test_statement_for_statement_oracle_small(device, oracle):
    rng = random.Random(3)
    q, r = _mutated_pairs(rng, 200, 80)
    cfg = WFAConfig(4, 6, 2, 200)
    ref = oracle_wfa(oracle, q, r, cfg, envelope=False)
    assert_same(device.wfa_affine(q, r, cfg), ref, "faithful oracle")


def test_edges(device, oracle):
    qs = ["", "", "A", "", "ACGT", "A" * 64, "A" * 65, "ACGT" * 40, "N" * 50, "A" * 33]
    rs = ["", "ACGT", "", "A" * 100, "ACGT", "A" * 65, "A" * 64, "TGCA" * 40, "A" * 50, "C" * 33]
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    for me in (0, 1, 8, 200, 1000):
        cfg = WFAConfig(4, 6, 2, me)
        assert_same(device.wfa_affine(q, r, cfg), oracle_wfa(oracle, q, r, cfg), f"me={me}")


def test_workload2_sample_exact_cover(device, oracle):
    q, r, _, _ = synth.generate(2, 3000)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    cfg = WFAConfig(4, 6, 2, me)
    ref = oracle_wfa(oracle, q, r, cfg)
    assert (ref >= 0).all()
    got = device.wfa_affine(q, r, cfg, batched=True)
    assert_same(got, ref, "workload 2")
    dq, dr = device.upload_batch(q), device.upload_batch(r)
    assert_same(device.wfa_affine(dq, dr, cfg, batched=False), ref, "workload 2 resident plain")


def test_workload2_max_error_200(device, oracle):
    q, r, _, _ = synth.generate(2, 2000, seed=12)
    cfg = WFAConfig(4, 6, 2, 200)
    ref = oracle_wfa(oracle, q, r, cfg)
    assert (ref == -1).any() and (ref >= 0).any()
    assert_same(device.wfa_affine(q, r, cfg), ref, "max_error 200")


def test_errors(device):
    q = SequenceBatch.from_strings(["ACGT"])
    r = SequenceBatch.from_strings(["ACGT"])
    for bad in (WFAConfig(0, 6, 2, 10), WFAConfig(4, 6, 0, 10), WFAConfig(4, -1, 2, 10),
                WFAConfig(4, 6, 2, -1), WFAConfig(100, 6, 1, 10)):
        with pytest.raises(GenomicsError):
            device.wfa_affine(q, r, bad)


def _random_seq(rng, n):
    return "".join(rng.choice("ACGT") for _ in range(n))


def _mutate(rng, q, rate):
    r = list(q)
    for _k in range(int(len(q) * rate)):
        pos = rng.randint(0, max(len(r) - 1, 0))
        op = rng.random()
        if op < 0.6 and r:
            r[pos] = rng.choice("ACGT")
        elif op < 0.8:
            r[pos:pos] = rng.choice("ACGT") * rng.randint(1, 4)
        elif r:
            del r[pos:pos + rng.randint(1, 4)]
    return "".join(r)


def test_length_classes(device, oracle):
    """Pairs on both sides of the block-per-pair threshold (2,048 bases), of
    the per-warp and per-block shared-memory sequence copies (10,240 and
    41,056 bases), unrelated pairs whose diagonal interval grows to thousands,
    and long pairs: batched, plain and tuning variants against the oracle.
    This batch (66 pairs, some of 8 kbp or more) runs the 16-warp kernel by
    default; the tuning variants run the 4-warp kernel."""
    rng = random.Random(2024)
    qs, rs = [], []
    for _ in range(40):                       # around the threshold, narrow intervals
        q = _random_seq(rng, rng.randint(1500, 3072))
        qs.append(q)
        rs.append(_mutate(rng, q, 0.05))
    for _ in range(6):                        # unrelated: interval > 1024
        qs.append(_random_seq(rng, rng.randint(2500, 3072)))
        rs.append(_random_seq(rng, rng.randint(2500, 3072)))
    for _ in range(12):                       # past the per-warp shared copies
        q = _random_seq(rng, rng.randint(3073, 20480))
        qs.append(q)
        rs.append(_mutate(rng, q, 0.03)[:20480])
    for _ in range(3):                        # unrelated: interval > 8192
        qs.append(_random_seq(rng, rng.randint(9000, 10000)))
        rs.append(_random_seq(rng, rng.randint(9000, 10000)))
    for _ in range(3):                        # long
        q = _random_seq(rng, rng.randint(20481, 24000))
        qs.append(q)
        rs.append(_mutate(rng, q, 0.02))
    for _ in range(2):                        # too long for a block's shared copies
        q = _random_seq(rng, rng.randint(41100, 45000))
        qs.append(q)
        rs.append(_mutate(rng, q, 0.01))
    order = list(range(len(qs)))
    rng.shuffle(order)
    q = SequenceBatch.from_strings([qs[i] for i in order])
    r = SequenceBatch.from_strings([rs[i] for i in order])
    for me in (3000, 24000):
        cfg = WFAConfig(4, 6, 2, me)
        ref = oracle_wfa(oracle, q, r, cfg)
        assert (ref >= 0).any()
        assert_same(device.wfa_affine(q, r, cfg, batched=True), ref, f"classes me={me}")
        assert_same(device.wfa_affine(q, r, cfg, batched=False), ref, f"plain me={me}")
        # every pair one warp each (no block-per-pair class), and a 4x threshold
        for v in (0x40, 0x80):
            assert_same(device.wfa_affine(q, r, cfg, batched=True, flags=v << 8), ref,
                        f"variant {v:#x} me={me}")
    # penalties with gcd 1 and 14 ring slots
    cfg = WFAConfig(5, 2, 3, 3000)
    ref = oracle_wfa(oracle, q, r, cfg)
    assert_same(device.wfa_affine(q, r, cfg, batched=True), ref, "(5,2,3)")


def test_int16_step_cap_rerun(device, oracle):
    """Queries of ~31.5 kbp whose alignments need more score steps than
    32767 - qlen: int16 rings give up at that step and the pair is run again
    with int32 rings; the costs equal the oracle's."""
    rng = random.Random(31)
    qs, rs = [], []
    for rate in (0.03, 0.04, 0.01):
        q = _random_seq(rng, rng.randint(31200, 31800))
        qs.append(q)
        rs.append(_mutate(rng, q, rate))
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    cfg = WFAConfig(4, 6, 2, 30000)
    ref = oracle_wfa(oracle, q, r, cfg)
    assert (ref >= 0).all() and (ref // 2 > 32767 - 31800).any()
    for batched in (True, False):
        assert_same(device.wfa_affine(q, r, cfg, batched=batched), ref, f"batched={batched}")


def test_bound_pruning_gives_the_same_costs(device, oracle):
    """Batches with long pairs run a bound pass (a banded WFA over the pairs the
    first tier suspends) and prune the later tiers by it; GB2_FLAG_NO_PRUNE turns
    both off.  Both equal the oracle, at the exact-cover budget and at budgets
    below some pairs' costs (-1), with penalty sets of other slot counts."""
    from genomics_b200._lib import FLAG_NO_PRUNE
    q, r, _, _ = synth.generate(2, 4000, seed=77)
    for pen in ((4, 6, 2), (2, 3, 1), (5, 2, 3)):
        for me in (synth.wfa_max_error_cover(q, r, *pen), 1500):
            cfg = WFAConfig(*pen, me)
            ref = oracle_wfa(oracle, q, r, cfg)
            for fl in (0, FLAG_NO_PRUNE):
                assert_same(device.wfa_affine(q, r, cfg, batched=True, flags=fl), ref,
                            f"{pen} me={me} flags={fl}")
