"""Gap-affine WFA with CIGAR traceback on the GPU (wfa_affine_cigar_cpu,
genomics/cpu/align_cpu.mojo:380-623) against the oracle: identical costs and
identical CIGAR strings, through the C ABI."""
import random

import numpy as np
import pytest

from genomics_b200 import SequenceBatch, WFAConfig, synth

pytestmark = pytest.mark.gpu

PENALTIES = [(4, 6, 2), (2, 3, 1), (1, 0, 1), (6, 4, 2), (3, 5, 2), (5, 2, 3)]


def _cigar_cost(cigar, x, o, e):
    """tests/test_alignment.mojo:145-166."""
    cost, cnt = 0, 0
    for ch in cigar:
        if ch.isdigit():
            cnt = cnt * 10 + int(ch)
        else:
            if ch == "X":
                cost += cnt * x
            elif ch in "ID":
                cost += o + cnt * e
            cnt = 0
    return cost


def _cigar_len(cigar, ops):
    tot, cnt = 0, 0
    for ch in cigar:
        if ch.isdigit():
            cnt = cnt * 10 + int(ch)
        else:
            if ch in ops:
                tot += cnt
            cnt = 0
    return tot


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


def _pairs(rng, n, maxlen):
    qs, rs = [], []
    for _ in range(n):
        q = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, maxlen)))
        r = _mutate(rng, q, rng.choice([0.0, 0.02, 0.1, 0.3])) if rng.random() < 0.85 else \
            "".join(rng.choice("ACGT") for _ in range(rng.randint(0, maxlen)))
        qs.append(q)
        rs.append(r)
    return qs, rs


def _check(device, oracle, qs, rs, pen, me, oracle_me=None):
    cfg = WFAConfig(*pen, me)
    cost, cig = device.wfa_cigar(SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs),
                                 cfg)
    for i, (q, r) in enumerate(zip(qs, rs)):
        ref_me = me if oracle_me is None else oracle_me[i]
        rc, rcig = oracle.wfa_cigar(q, r, *pen, ref_me)
        if oracle_me is not None and rc == -1:
            continue  # the GPU ran with a larger budget; only compare found costs
        assert (int(cost[i]), cig[i]) == (rc, rcig), (pen, me, i, len(q), len(r))


def test_known_answers(device, known):
    cfg = WFAConfig(4, 6, 2, 200)
    for case in known["wfa_cigar"]:
        qb = SequenceBatch.from_strings([case["q"]])
        rb = SequenceBatch.from_strings([case["r"]])
        qp, _, _, ql = qb.arrays()
        rp, _, _, rl = rb.arrays()
        assert device.wfa_cigar_pair(qp, int(ql[0]), rp, int(rl[0]), cfg) == \
            (case["cost"], case["cigar"]), case["src"]
    cases = known["wfa_cigar"]
    cost, cig = device.wfa_cigar(SequenceBatch.from_strings([c["q"] for c in cases]),
                                 SequenceBatch.from_strings([c["r"] for c in cases]), cfg)
    assert [(int(a), b) for a, b in zip(cost, cig)] == [(c["cost"], c["cigar"]) for c in cases]


def test_consistency_pairs(device, oracle, known):
    qs = [q for q, _ in known["wfa_cigar_consistency"]["pairs"]]
    rs = [r for _, r in known["wfa_cigar_consistency"]["pairs"]]
    cost, cig = device.wfa_cigar(SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs),
                                 WFAConfig(4, 6, 2, 200))
    for q, r, c, s in zip(qs, rs, cost, cig):
        assert c == oracle.wfa_affine(q, r)
        assert _cigar_cost(s, 4, 6, 2) == c
        assert _cigar_len(s, "=XI") == len(q) and _cigar_len(s, "=XD") == len(r)


def test_edges(device, oracle):
    qs = ["", "", "ACGT", "A", "ACGT", "ACGTACGT" * 8, "A" * 33, "N" * 20]
    rs = ["", "ACGT", "", "", "ACGT", "ACGTACGT" * 8, "C" * 33, "A" * 20]
    for me in (0, 1, 8, 40, 300):
        _check(device, oracle, qs, rs, (4, 6, 2), me)


@pytest.mark.parametrize("pen", PENALTIES)
def test_random_pairs(device, oracle, pen):
    rng = random.Random(sum(pen) * 7 + 1)
    qs, rs = _pairs(rng, 160, 160)
    for me in (0, 12, 60, 400):
        _check(device, oracle, qs, rs, pen, me)


def test_longer_pairs(device, oracle):
    """Pairs of 500-2,500 bases (several warps' worth of diagonals per score)
    and unrelated pairs; the oracle runs with max_error = the exact cost
    (its arrays grow with max_error^2), the GPU with a larger budget, which
    leaves cost and CIGAR unchanged."""
    rng = random.Random(5)
    qs, rs = [], []
    for _ in range(24):
        q = "".join(rng.choice("ACGT") for _ in range(rng.randint(500, 2500)))
        qs.append(q)
        rs.append(_mutate(rng, q, rng.choice([0.01, 0.03, 0.05])))
    for _ in range(3):
        qs.append("".join(rng.choice("ACGT") for _ in range(rng.randint(300, 500))))
        rs.append("".join(rng.choice("ACGT") for _ in range(rng.randint(300, 500))))
    exact = [oracle.wfa_affine(q, r, 4, 6, 2, 6000, envelope=True) for q, r in zip(qs, rs)]
    assert all(c >= 0 for c in exact)
    _check(device, oracle, qs, rs, (4, 6, 2), 6000, oracle_me=exact)


def test_long_workload_properties(device):
    """2,000 pairs of the long-pair workload (100-10,000 bp): the CIGAR's cost
    equals the cost kernel's, and it consumes both sequences exactly."""
    q, r, _, _ = synth.generate(2, 2000, seed=21)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    cfg = WFAConfig(4, 6, 2, me)
    cost, cig = device.wfa_cigar(q, r, cfg)
    ref = device.wfa_affine(q, r, cfg)
    assert (cost == ref).all() and (cost >= 0).all()
    _, _, _, ql = q.arrays()
    _, _, _, rl = r.arrays()
    for i in range(len(cig)):
        assert _cigar_cost(cig[i], 4, 6, 2) == cost[i]
        assert _cigar_len(cig[i], "=XI") == ql[i] and _cigar_len(cig[i], "=XD") == rl[i]


def test_runs_capacity_error(device):
    """A runs array that is too small: GB2_ERANGE and the count needed."""
    import ctypes
    from genomics_b200._lib import GB2_ERANGE
    from genomics_b200.device import _ptr, _wfa_cfg
    q = device.upload_batch(SequenceBatch.from_strings(["ACGTACGTAC", "AAAA"]), with_nmask=False)
    r = device.upload_batch(SequenceBatch.from_strings(["ACGAACGTTC", "AATA"]), with_nmask=False)
    cost = np.zeros(2, np.int32)
    offs = np.zeros(3, np.int64)
    runs = np.zeros(1, np.uint32)
    rc = device.L.gb2_wfa_cigar(device.ctx, q.handle, r.handle,
                                ctypes.byref(_wfa_cfg(WFAConfig(4, 6, 2, 100))), 2, _ptr(cost),
                                _ptr(runs), 1, _ptr(offs), 0)
    assert rc == GB2_ERANGE and offs[2] > 1
    q.close()
    r.close()


def test_cigar_after_int32_rerun(device):
    """A ~31.5 kbp pair run again with int32 rings in the CIGAR pass: its
    CIGAR re-scores to the cost and consumes both sequences."""
    rng = random.Random(32)
    q = "".join(rng.choice("ACGT") for _ in range(31500))
    r = _mutate(rng, q, 0.03)
    cfg = WFAConfig(4, 6, 2, 30000)
    cost, cig = device.wfa_cigar(SequenceBatch.from_strings([q]), SequenceBatch.from_strings([r]),
                                 cfg)
    assert cost[0] == device.wfa_affine(SequenceBatch.from_strings([q]),
                                        SequenceBatch.from_strings([r]), cfg)[0]
    assert cost[0] // 2 > 32767 - 31500
    assert _cigar_cost(cig[0], 4, 6, 2) == cost[0]
    assert _cigar_len(cig[0], "=XI") == len(q) and _cigar_len(cig[0], "=XD") == len(r)


def test_grouped_arena_matches_one_group(device):
    """A history arena capped at 2 MiB (GB2_FLAGS_ARENA_MIB) splits these pairs
    into several groups; costs and CIGARs equal those of one group."""
    rng = random.Random(77)
    qs, rs = [], []
    for _ in range(24):
        q = "".join(rng.choice("ACGT") for _ in range(rng.randint(500, 2500)))
        qs.append(q)
        rs.append(_mutate(rng, q, rng.choice([0.01, 0.03, 0.05])))
    qb, rb = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    cfg = WFAConfig(4, 6, 2, 6000)
    one = device.wfa_cigar(qb, rb, cfg)
    grouped = device.wfa_cigar(qb, rb, cfg, flags=2 << 24)
    assert (one[0] == grouped[0]).all() and list(one[1]) == list(grouped[1])
    assert (one[0] >= 0).all()
