"""Banded Smith-Waterman on the GPU against the oracle: bit-exact scores and
end cells (score, query_end, ref_end), through the C ABI."""
import random

import numpy as np
import pytest

import genomics_b200 as G
from genomics_b200 import AlignConfig, SequenceBatch, synth
from genomics_b200._lib import FLAG_GENERIC, FLAG_INT32, FLAG_PACKED, GenomicsError

pytestmark = pytest.mark.gpu

CFG0 = AlignConfig(2, -4, -4, -2, 32)  # scoring of the read workloads


def oracle_sw(O, q, r, cfg, bands=None, n=None):
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    if n is not None:
        qo, ql, ro, rl = qo[:n], ql[:n], ro[:n], rl[:n]
        if bands is not None:
            bands = np.asarray(bands)[:n]
    return O.sw_batch(qp, qo, ql, rp, ro, rl, cfg.match_score, cfg.mismatch, cfg.gap_open,
                      cfg.gap_extend, cfg.band_width, bands=bands)


def assert_same(got, ref, what=""):
    sc, qe, re_ = ref
    bad = np.nonzero((got["score"] != sc) | (got["query_end"] != qe) | (got["ref_end"] != re_))[0]
    assert bad.size == 0, (f"{what}: {bad.size} mismatches, first {bad[:5]} "
                           f"got {got[bad[:3]]} want {[(sc[i], qe[i], re_[i]) for i in bad[:3]]}")


def subset(b: SequenceBatch, idx):
    p, m, o, l = b.arrays()
    seqs_p, seqs_m, offs, lens = [], [], [], []
    w = 0
    for i in idx:
        nw = (int(l[i]) + 31) // 32
        seqs_p.append(p[o[i]:o[i] + nw])
        seqs_m.append(m[o[i]:o[i] + nw])
        offs.append(w)
        lens.append(int(l[i]))
        w += nw
    cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0, np.uint64)
    return SequenceBatch.from_arrays(cat(seqs_p), cat(seqs_m), np.array(offs, np.int64),
                                     np.array(lens, np.int64))


def test_known_answers_dropin(device, known):
    d = G.default_config()
    for case in known["sw"]:
        qb = SequenceBatch.from_strings([case["q"]])
        rb = SequenceBatch.from_strings([case["r"]])
        cfg = AlignConfig(d.match_score, d.mismatch, d.gap_open, d.gap_extend, case["band"])
        res = G.smith_waterman_banded(G.get_view(qb, 0), G.get_view(rb, 0), cfg)
        if "score" in case:
            assert res.score == case["score"], case["src"]
        else:
            assert res.score >= case["score_at_least"], case["src"]
        assert res.query_start == 0 and res.ref_start == 0 and res.cigar == []


def _random_pairs(rng, n, maxlen, alphabet="ACGT"):
    qs, rs = [], []
    for _ in range(n):
        q = "".join(rng.choice(alphabet) for _ in range(rng.randint(0, maxlen)))
        if q and rng.random() < 0.6:
            r = list(q[rng.randint(0, len(q) // 3):])
            for _k in range(rng.randint(0, 6)):
                pos = rng.randint(0, max(len(r) - 1, 0))
                op = rng.random()
                if op < 0.5 and r:
                    r[pos] = rng.choice("ACGT")
                elif op < 0.75:
                    r.insert(pos, rng.choice("ACGT"))
                elif r:
                    del r[pos]
            r = "".join(r) + "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 20)))
        else:
            r = "".join(rng.choice(alphabet) for _ in range(rng.randint(0, maxlen)))
        qs.append(q)
        rs.append(r)
    return SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)


@pytest.mark.parametrize("band", [16, 32, 64, 128, 0, 1, 5, 31, 40])
def test_random_pairs_all_paths(device, oracle, band):
    rng = random.Random(100 + band)
    q, r = _random_pairs(rng, 600, 300, "ACGTN")
    for cfg in (AlignConfig(2, -4, -4, -2, band), AlignConfig(2, -3, -5, -2, band),
                AlignConfig(1, -1, 0, -1, band), AlignConfig(5, 0, -2, 0, band)):
        ref = oracle_sw(oracle, q, r, cfg)
        for batched in (False, True):
            assert_same(device.sw_banded(q, r, cfg, batched=batched), ref,
                        f"band {band} cfg {cfg} batched {batched}")
        assert_same(device.sw_banded(q, r, cfg, flags=FLAG_GENERIC), ref, "literal kernel")


def test_out_of_domain_configs_use_literal_kernel(device, oracle):
    rng = random.Random(5)
    q, r = _random_pairs(rng, 300, 120)
    for cfg in (AlignConfig(2, -4, 3, -1, 32), AlignConfig(2, -4, -4, 1, 16),
                AlignConfig(2, 1, -4, -2, 64), AlignConfig(-1, -4, -4, -2, 32)):
        ref = oracle_sw(oracle, q, r, cfg)
        assert_same(device.sw_banded(q, r, cfg, batched=True), ref, f"cfg {cfg}")


def test_edge_lengths(device, oracle):
    lens = [0, 1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129, 1023, 1024, 1025]
    rng = random.Random(9)
    qs, rs = [], []
    for a in lens:
        for b in lens:
            base = "".join(rng.choice("ACGT") for _ in range(max(a, b)))
            qs.append(base[:a])
            rs.append(base[:b] if rng.random() < 0.5 else "".join(rng.choice("ACGT") for _ in range(b)))
    qs += ["N" * 100, "ACGT" * 50, "A" * 300]
    rs += ["A" * 100, "N" * 200, "A" * 5]
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    for band in (16, 32, 64, 128, 3):
        cfg = AlignConfig(2, -4, -4, -2, band)
        ref = oracle_sw(oracle, q, r, cfg)
        assert_same(device.sw_banded(q, r, cfg, batched=True), ref, f"band {band}")
        assert_same(device.sw_banded(q, r, cfg, batched=False), ref, f"band {band} plain")


def test_long_pair_32k_boundary(device, oracle):
    rng = random.Random(2)
    base = "".join(rng.choice("ACGT") for _ in range(32800))
    qs = [base[:32767], base[:32768], base[5:32774]]
    rs = [base[:32768], base[3:32771], base[:32769]]
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    cfg = AlignConfig(2, -4, -4, -2, 32)
    assert_same(device.sw_banded(q, r, cfg), oracle_sw(oracle, q, r, cfg), "32k")


def test_workload0_full(device, oracle):
    q, r, bands, _ = synth.generate(0, 1000)
    ref = oracle_sw(oracle, q, r, CFG0)
    for batched in (False, True):
        assert_same(device.sw_banded(q, r, CFG0, batched=batched), ref, "workload 0")


def test_workload1_resident_subset_and_properties(device, oracle):
    q, r, bands, _ = synth.generate(1, 1_000_000)
    dq, dr = device.upload_batch(q), device.upload_batch(r)
    got = device.sw_banded(dq, dr, CFG0, batched=True)
    plain = device.sw_banded(dq, dr, CFG0, batched=False)
    assert (got == plain).all()
    # end to end from the host arrays (chunked pipeline)
    assert (device.sw_banded(q, r, CFG0) == got).all()
    # size-independent properties over all 1e6 pairs
    assert (got["score"] >= 0).all() and (got["score"] <= 2 * 150).all()
    assert (got["query_end"] < 150).all() and (got["ref_end"] < 200).all()
    assert (np.abs(got["ref_end"] - got["query_end"] - 0) <= 200).all()
    zero = got["score"] == 0
    assert (got["query_end"][zero] == 0).all() and (got["ref_end"][zero] == 0).all()
    # bit-exact on a seeded random sample of 40k pairs
    idx = np.sort(np.random.default_rng(1).choice(1_000_000, 40_000, replace=False))
    qs, rs = subset(q, idx), subset(r, idx)
    ref = oracle_sw(oracle, qs, rs, CFG0)
    assert_same(got[idx], ref, "workload 1 sample")
    dq.close()
    dr.close()


def test_workload3_mixed_bands(device, oracle):
    q, r, bands, _ = synth.generate(3, 6000)
    ref = oracle_sw(oracle, q, r, CFG0, bands=bands)
    for batched in (True, False):
        assert_same(device.sw_banded(q, r, CFG0, bands=bands, batched=batched), ref,
                    f"workload 3 batched={batched}")
    dq, dr = device.upload_batch(q), device.upload_batch(r)
    assert_same(device.sw_banded(dq, dr, CFG0, bands=bands), ref, "workload 3 resident")


@pytest.mark.parametrize("band", [16, 32])
def test_packed_int16_path_matches_int32_and_oracle(device, oracle, band):
    """Short pairs (H bound <= 511) take the packed int16x2 kernel by default;
    GB2_FLAG_INT32 forces the int32 register kernel.  Both equal the oracle."""
    rng = random.Random(band * 7)
    q, r = _random_pairs(rng, 3000, 255, "ACGTN")
    for cfg in (AlignConfig(2, -4, -4, -2, band), AlignConfig(1, -1, 0, -1, band),
                AlignConfig(3, -2, -6, -1, band), AlignConfig(2, -8, -2, -1, band)):
        ref = oracle_sw(oracle, q, r, cfg)
        for batched in (False, True):
            assert_same(device.sw_banded(q, r, cfg, batched=batched), ref, f"{cfg} packed")
            assert_same(device.sw_banded(q, r, cfg, batched=batched, flags=FLAG_INT32), ref,
                        f"{cfg} int32")
    q, r, _, _ = synth.generate(0, 1000, seed=99)
    cfg = AlignConfig(2, -4, -4, -2, band)
    ref = oracle_sw(oracle, q, r, cfg)
    assert_same(device.sw_banded(q, r, cfg), ref, "reads packed")
    assert_same(device.sw_banded(q, r, cfg, flags=FLAG_INT32), ref, "reads int32")


@pytest.mark.parametrize("band", [16, 32, 64, 128])
def test_packed_wide_keys_match_int32_and_oracle(device, oracle, band):
    """Pairs whose scores pass 511 (the narrow keys' limit) but stay within
    match * (min(qlen, rlen) + 1) <= 4094 take the packed kernel with group keys
    (GB2_FLAG_PACKED: these batches are small enough to run the int32 kernels by
    default, which must give the same results); GB2_FLAG_INT32 forces the int32
    register kernels.  All equal the oracle, including first-maximum ties across
    groups and halves and rows past either end."""
    rng = random.Random(band * 13)
    q, r = _random_pairs(rng, 600, 2000, "ACGTN")
    # similar pairs reach large scores; repeats make equal maxima in many columns
    reps = ["ACGT" * rng.randint(100, 450) for _ in range(40)]
    q2 = SequenceBatch.from_strings(reps + [s[:rng.randint(300, len(s))] for s in reps])
    r2 = SequenceBatch.from_strings([s[rng.randint(0, 20):] for s in reps] + reps)
    for qq, rr in ((q, r), (q2, r2)):
        for cfg in (AlignConfig(2, -4, -4, -2, band), AlignConfig(1, -1, 0, -1, band),
                    AlignConfig(3, -2, -6, -1, band), AlignConfig(2, -8, -2, -1, band)):
            ref = oracle_sw(oracle, qq, rr, cfg)
            for batched in (False, True):
                assert_same(device.sw_banded(qq, rr, cfg, batched=batched, flags=FLAG_PACKED),
                            ref, f"{cfg} wide packed batched={batched}")
            assert_same(device.sw_banded(qq, rr, cfg), ref, f"{cfg} default")
            assert_same(device.sw_banded(qq, rr, cfg, flags=FLAG_INT32), ref, f"{cfg} int32")


def test_packed_wide_key_bounds(device, oracle):
    """Pairs on both sides of the wide keys' score bound (match * (min + 1) =
    4094 at match 2: min length 2046), mixed bands per pair."""
    rng = random.Random(4094)
    qs, rs, bands = [], [], []
    for L in (2044, 2045, 2046, 2047, 2048, 3000):
        for _ in range(4):
            s = "".join(rng.choice("ACGT") for _ in range(L))
            qs.append(s)
            rs.append(s[:L // 2] + "G" + s[L // 2 + 1:])
            bands.append(rng.choice([16, 32, 64, 128]))
    q, r = SequenceBatch.from_strings(qs), SequenceBatch.from_strings(rs)
    b = np.array(bands, np.int32)
    ref = oracle_sw(oracle, q, r, CFG0, bands=b)
    assert (ref[0] > 4000).any()
    for batched in (False, True):
        for flags in (0, FLAG_PACKED):
            assert_same(device.sw_banded(q, r, CFG0, bands=b, batched=batched, flags=flags),
                        ref, f"bounds batched={batched} flags={flags}")


def test_variants_agree(device, oracle):
    q, r, bands, _ = synth.generate(3, 3000, seed=77)
    ref = oracle_sw(oracle, q, r, CFG0, bands=bands)
    for v in (1, 2):
        assert_same(device.sw_banded(q, r, CFG0, bands=bands, flags=v << 8), ref, f"variant {v}")


def test_reference_harness_pairs(device, oracle):
    """The reference's own benchmark input (identical LCG pairs, 500 bp)."""
    q, r, _, _ = synth.generate(100, 100, param=500)
    for band in (16, 32, 64, 128):
        cfg = AlignConfig(2, -3, -5, -2, band)
        got = device.sw_banded(q, r, cfg)
        assert_same(got, oracle_sw(oracle, q, r, cfg), f"harness band {band}")
        assert (got["score"] == 1000).all()


def test_errors(device):
    q = SequenceBatch.from_strings(["ACGT"])
    r = SequenceBatch.from_strings(["ACGT"])
    with pytest.raises(GenomicsError):
        device.sw_banded(q, r, AlignConfig(2, -4, -4, -2, -1))
    with pytest.raises(GenomicsError):
        device.sw_banded(q, r, AlignConfig(200_000_000, -4, -4, -2, 32))
    dq = device.upload_batch(q)
    dr = device.upload_batch(r)
    with pytest.raises(GenomicsError):
        device.sw_banded(dq, dr, CFG0, n_pairs=2)
    assert device.sw_banded(dq, dr, CFG0, n_pairs=0).size == 0


def test_device_packing_matches_add_sequence(device, oracle):
    """gb2_batch_from_ascii packs on the GPU exactly as add_sequence does."""
    rng = random.Random(31)
    seqs = ["", "A", "N", "ACGT" * 8, "acgtNNRYacgt", "T" * 33, "G" * 64, "C" * 65]
    seqs += ["".join(rng.choice("ACGTNacgtn-RYKM") for _ in range(rng.randint(0, 700)))
             for _ in range(400)]
    got = device.download_batch(device.batch_from_ascii(seqs))
    want = SequenceBatch.from_strings(seqs)
    for x, y in zip(got.arrays(), want.arrays()):
        assert (x == y).all()
    for i, s in enumerate(seqs[:60]):
        op, om = oracle.pack(s)
        o, nw = int(got.offsets[i]), (len(s) + 31) // 32
        assert (got.packed[o:o + nw] == op).all() and (got.n_masks[o:o + nw] == om).all()
    # and a device-packed batch aligns like a host-packed one
    q, r, bands, _ = synth.generate(3, 500, seed=8)
    qs = ["".join("ACGT"[(int(w) >> (62 - 2 * j)) & 3] if not (int(m) >> j) & 1 else "N"
                  for w, m in zip(q.packed[q.offsets[i]:q.offsets[i] + (q.lengths[i] + 31) // 32],
                                  q.n_masks[q.offsets[i]:q.offsets[i] + (q.lengths[i] + 31) // 32])
                  for j in range(32))[:q.lengths[i]] for i in range(500)]
    dq = device.batch_from_ascii(qs)
    dr = device.upload_batch(r)
    assert_same(device.sw_banded(dq, dr, CFG0, bands=bands), oracle_sw(oracle, q, r, CFG0, bands=bands),
                "device-packed queries")


def _permuted_layout(b: SequenceBatch, rng):
    """The same sequences stored in a shuffled order of the word array, with
    one gap word between them: offsets no longer ascend."""
    p, m, o, l = b.arrays()
    perm = list(range(len(l)))
    rng.shuffle(perm)
    words, masks, offs = [], [], np.zeros(len(l), np.int64)
    w = 0
    for i in perm:
        nw = (int(l[i]) + 31) // 32
        offs[i] = w
        words.append(p[o[i]:o[i] + nw])
        masks.append(m[o[i]:o[i] + nw])
        words.append(np.zeros(1, np.uint64))
        masks.append(np.zeros(1, np.uint64))
        w += nw + 1
    return SequenceBatch.from_arrays(np.concatenate(words), np.concatenate(masks), offs,
                                     l.copy())


def test_host_pipeline_layouts_and_chunks(device, oracle):
    """The host entry point over any layout (shuffled offsets, gaps, one
    sequence shared by several pairs), split into 1..many chunks, equals the
    resident path and the oracle; a bad length in a late chunk is an error
    that leaves the context usable."""
    rng = random.Random(77)
    q, r = _random_pairs(rng, 3000, 300)
    cfg = AlignConfig(2, -4, -4, -2, 24)
    ref = oracle_sw(oracle, q, r, cfg)
    qs, rs = _permuted_layout(q, rng), _permuted_layout(r, rng)
    for ch in (0, 1, 3, 7, 64):
        assert_same(device.sw_banded(qs, rs, cfg, flags=ch << 16), ref, f"chunks {ch}")
    # pairs 10..19 all use the reference sequence of pair 10
    p, m, o, l = rs.arrays()
    o2, l2 = o.copy(), l.copy()
    o2[10:20], l2[10:20] = o[10], l[10]
    shared = SequenceBatch.from_arrays(p, m, o2, l2)
    got = device.sw_banded(qs, shared, cfg, flags=5 << 16)
    ref2 = oracle_sw(oracle, q, SequenceBatch.from_arrays(p, m, o2, l2), cfg)
    assert_same(got, ref2, "shared sequence")
    # a negative length among the last pairs: error, then a clean call
    bad_l = l.copy()
    bad_l[-3] = -1
    with pytest.raises(GenomicsError):
        device.sw_banded(qs, SequenceBatch.from_arrays(p, m, o, bad_l), cfg, flags=4 << 16)
    assert_same(device.sw_banded(qs, rs, cfg, flags=4 << 16), ref, "after the error")
