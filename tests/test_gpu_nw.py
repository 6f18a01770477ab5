"""Banded Needleman-Wunsch on the GPU (needleman_wunsch_banded with the band
rows sized as genomics/cpu/align_cpu.mojo:327-341 index them) against the
oracle: identical scores and end cells, register and literal kernels."""
import random

import numpy as np
import pytest

import genomics_b200 as G
from genomics_b200 import AlignConfig, SequenceBatch, synth
from genomics_b200._lib import FLAG_GENERIC, GenomicsError

pytestmark = pytest.mark.gpu

SCORINGS = [(2, -3, -5, -2), (2, -4, -4, -2), (1, -1, -2, -1), (3, -2, -3, 0), (2, 1, 2, -1)]


def oracle_nw(O, q, r, cfg, bands=None):
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    return O.nw_batch(qp, qo, ql, rp, ro, rl, cfg.match_score, cfg.mismatch, cfg.gap_open,
                      cfg.gap_extend, cfg.band_width, bands=bands)


def check(got, ref, q, r, what):
    _, _, _, ql = q.arrays()
    _, _, _, rl = r.arrays()
    bad = np.nonzero(got["score"] != ref)[0]
    assert bad.size == 0, f"{what}: {bad.size} mismatches, first {bad[:5]} got " \
                          f"{got['score'][bad[:5]]} want {ref[bad[:5]]}"
    assert (got["query_end"] == ql - 1).all() and (got["ref_end"] == rl - 1).all()


def _pairs(rng, n, maxlen):
    qs, rs = [], []
    for _ in range(n):
        q = "".join(rng.choice("ACGTN") for _ in range(rng.randint(0, maxlen)))
        if rng.random() < 0.7:
            r = list(q)
            for _k in range(rng.randint(0, max(1, len(q) // 8))):
                pos = rng.randint(0, max(len(r) - 1, 0))
                op = rng.random()
                if op < 0.6 and r:
                    r[pos] = rng.choice("ACGT")
                elif op < 0.8:
                    r[pos:pos] = rng.choice("ACGT") * rng.randint(1, 3)
                elif r:
                    del r[pos:pos + rng.randint(1, 3)]
            r = "".join(r)
        else:
            r = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, maxlen)))
        qs.append(q)
        rs.append(r)
    return SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)


def test_known_answers_dropin(device, known):
    d = G.default_config()
    for case in known["nw"]:
        qb = SequenceBatch.from_strings([case["q"]])
        rb = SequenceBatch.from_strings([case["r"]])
        cfg = AlignConfig(d.match_score, d.mismatch, d.gap_open, d.gap_extend, case["band"])
        res = G.needleman_wunsch_banded(G.get_view(qb, 0), G.get_view(rb, 0), cfg)
        assert res.score == case["score"], case["src"]
        assert (res.query_end, res.ref_end) == (len(case["q"]) - 1, len(case["r"]) - 1)


@pytest.mark.parametrize("band", [0, 1, 5, 16, 31, 32, 40, 64])
def test_random_pairs(device, oracle, band):
    rng = random.Random(band + 11)
    q, r = _pairs(rng, 500, 260)
    for sc in SCORINGS:
        cfg = AlignConfig(*sc, band)
        ref = oracle_nw(oracle, q, r, cfg)
        check(device.nw_banded(q, r, cfg), ref, q, r, f"band {band} {sc}")
        check(device.nw_banded(q, r, cfg, flags=FLAG_GENERIC), ref, q, r, f"literal {band} {sc}")


def test_per_pair_bands(device, oracle):
    rng = random.Random(3)
    q, r = _pairs(rng, 600, 300)
    bands = np.array([rng.choice([0, 3, 16, 32, 50, 128]) for _ in range(600)], np.int32)
    cfg = AlignConfig(2, -3, -5, -2, 32)
    check(device.nw_banded(q, r, cfg, bands=bands), oracle_nw(oracle, q, r, cfg, bands), q, r,
          "per-pair bands")


def test_read_workload(device, oracle):
    """The 1,000-pair read workload (150 bp vs 200 bp): the final cell lies
    50 diagonals off, outside band 32 (score -1000000), inside band 64."""
    q, r, _, _ = synth.generate(0, 1000)
    for band in (32, 16):
        cfg = AlignConfig(2, -4, -4, -2, band)
        check(device.nw_banded(q, r, cfg), oracle_nw(oracle, q, r, cfg), q, r, f"reads {band}")
    cfg = AlignConfig(2, -4, -4, -2, 64)
    ref = oracle_nw(oracle, q, r, cfg)
    assert (ref > -1000000).all()
    check(device.nw_banded(q, r, cfg), ref, q, r, "reads 64")


def test_equal_length_pairs_register_kernel(device, oracle):
    """Equal-length mutated pairs up to 2,000 bp, band 32: the register kernel
    over rows where every cell is inside the matrix, against the oracle."""
    rng = random.Random(9)
    qs, rs = [], []
    for _ in range(2000):
        L = rng.randint(1, 2000)
        a = "".join(rng.choice("ACGT") for _ in range(L))
        b = "".join(c if rng.random() > 0.05 else rng.choice("ACGT") for c in a)
        qs.append(a)
        rs.append(b)
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    cfg = AlignConfig(2, -4, -4, -2, 32)
    check(device.nw_banded(q, r, cfg), oracle_nw(oracle, q, r, cfg), q, r, "equal length")


def test_errors(device):
    q = SequenceBatch.from_strings(["ACGT"])
    with pytest.raises(GenomicsError):
        device.nw_banded(q, q, AlignConfig(2, -3, -5, -2, -1))
    with pytest.raises(GenomicsError):
        device.nw_banded(q, q, AlignConfig(2, -3, -5, -2, 4), bands=np.array([-2], np.int32))
    big = AlignConfig(200_000_000, -3, -5, -2, 4)
    with pytest.raises(GenomicsError):
        device.nw_banded(q, q, big)
