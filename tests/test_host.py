"""Host-side mirror of the reference's core types (genomics/core/*.mojo) and the
synthetic workload generator.  CPU only."""
import numpy as np
import pytest

import genomics_b200 as G
from genomics_b200 import synth


def test_ascii_to_2bit(known):
    for c, v in known["encoding"]["ascii_to_2bit"]["cases"]:
        assert G.ascii_to_2bit(c) == v
    for b in range(4):  # tests/test_dna.mojo:25-28
        assert G.ascii_to_2bit(G.base_to_ascii(b)) == b


def test_get_base_from_word(known):
    g = known["encoding"]["get_base_from_word"]
    w = int(g["word_hex"], 16)
    assert [G.get_base_from_word(w, i) for i in range(5)] == g["bases"]


def test_nmask(known):
    nm = G.NMask.empty()
    assert not nm.has_any_n()
    nm.set_n(0)
    assert nm.is_n(0) and not nm.is_n(1) and nm.has_any_n()
    nm.set_n(31)
    assert nm.is_n(31) and nm.any_n_in_range(0, 32) and not nm.any_n_in_range(1, 31)
    g = known["encoding"]["nmask"]
    nm = G.NMask.empty()
    for p in g["set"]:
        nm.set_n(p)
    for a, b in g["true_ranges"]:
        assert nm.any_n_in_range(a, b)
    for a, b in g["false_ranges"]:
        assert not nm.any_n_in_range(a, b)


def test_sequence_batch(known):
    enc = known["encoding"]
    b = G.SequenceBatch.from_strings(["ACGT", "TTTT", "AAAA"])
    assert b.count == 3
    assert G.SequenceBatch.from_strings(enc["batch_total"]["seqs"]).total_bases() == 12
    v = G.get_view(G.SequenceBatch.from_strings([enc["view_bases"]["seq"]]), 0)
    assert v.length == 4 and [v.get_base(i) for i in range(4)] == enc["view_bases"]["bases"]
    v = G.get_view(G.SequenceBatch.from_strings([enc["view_33"]["seq"]]), 0)
    assert v.length == 33 and v.word_count == 2 and v.get_base(32) == 0
    v = G.get_view(G.SequenceBatch.from_strings([enc["n_tracking"]["seq"]]), 0)
    assert [v.is_n(i) for i in range(4)] == enc["n_tracking"]["is_n"]
    v = G.get_view(G.SequenceBatch.from_strings([enc["n_window"]["seq"]]), 0)
    for a, c in enc["n_window"]["true"]:
        assert v.has_n_in_window(a, c)
    for a, c in enc["n_window"]["false"]:
        assert not v.has_n_in_window(a, c)
    b = G.SequenceBatch.from_strings(enc["batch_independent"]["seqs"])
    for i in range(4):
        v = G.get_view(b, i)
        assert [v.get_base(j) for j in range(4)] == [i] * 4


def test_pack_matches_oracle(oracle):
    rng = np.random.default_rng(3)
    seqs = []
    for _ in range(200):
        n = int(rng.integers(0, 130))
        seqs.append("".join(rng.choice(list("ACGTNacgtn-RY"), n)))
    seqs += ["", "A" * 32, "C" * 33, "G" * 64, "T" * 65]
    p, m, o, l = G.pack_ascii(seqs)
    for i, s in enumerate(seqs):
        op, om = oracle.pack(s)
        nw = (len(s) + 31) // 32
        assert (p[o[i]:o[i] + nw] == op).all() and (m[o[i]:o[i] + nw] == om).all()
        assert l[i] == len(s)
    # append layout: each sequence starts where the previous one ended
    assert (o[1:] == o[:-1] + (l[:-1] + 31) // 32).all()


def test_add_sequence_incremental_equals_bulk():
    seqs = ["ACGT" * 9, "NNAC", "", "acgtACGT"]
    a = G.SequenceBatch()
    for s in seqs:
        a.add_sequence(s, len(s))
    b = G.SequenceBatch.from_strings(seqs)
    for x, y in zip(a.arrays(), b.arrays()):
        assert (x == y).all()


@pytest.mark.parametrize("wl,n", [(0, 500), (2, 60), (3, 200), (4, 100), (100, 7)])
def test_generator_deterministic_and_shaped(wl, n):
    q1, r1, b1, k1 = synth.generate(wl, n)
    q2, r2, b2, k2 = synth.generate(wl, n)
    for x, y in zip(q1.arrays() + r1.arrays(), q2.arrays() + r2.arrays()):
        assert (x == y).all()
    assert (b1 == b2).all() and (k1 == k2).all()
    ql, rl = q1.lengths, r1.lengths
    assert ql.size == n and rl.size == n
    if wl == 0:
        assert (ql == 150).all() and (rl == 200).all() and (b1 == 32).all()
        assert not q1.n_masks.any() and not r1.n_masks.any()
    if wl == 2:
        assert ql.min() >= 100 and ql.max() <= 10000
    if wl == 3:
        assert ql.min() >= 100 and ql.max() <= 2000
        assert (rl == np.floor(1.25 * ql + 0.5)).all()  # llround: half away from zero
        assert set(np.unique(b1)) <= {16, 32, 64, 128}
    if wl == 100:
        # the reference harness aligns each LCG sequence with itself
        assert (q1.packed == r1.packed).all()


def test_generator_n_runs_stored_as_a():
    q, r, _, _ = synth.generate(3, 400)
    nm = q.n_masks
    frac = sum(bin(int(w)).count("1") for w in nm) / q.lengths.sum()
    assert 0.003 < frac < 0.02  # about 1% of positions in N runs
    # every N position holds code A (0) in the packed word
    for w, m in zip(q.packed[:2000], nm[:2000]):
        for i in range(32):
            if (int(m) >> i) & 1:
                assert (int(w) >> (62 - 2 * i)) & 3 == 0


def test_max_error_cover():
    q, r, _, _ = synth.generate(2, 50)
    ql, rl = q.lengths, r.lengths
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    i = int(np.argmax(4 * np.minimum(ql, rl) + np.where(ql != rl, 6 + 2 * abs(ql - rl), 0)))
    assert me == 4 * min(ql[i], rl[i]) + (6 + 2 * abs(int(ql[i]) - int(rl[i])) if ql[i] != rl[i] else 0)


def test_sw_cells_convention():
    q, r, b, _ = synth.generate(0, 10)
    assert synth.sw_cells(q, b) == 10 * 150 * 65


def test_bench_window_batch_matches_slicing():
    """bench.py's NW workload: bases [25, 175) of each 200 bp target, repacked."""
    import sys
    from conftest import ROOT
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    from genomics_b200 import synth
    _, r, _, _ = synth.generate(1, 300, seed=3)
    w = bench._window_batch(r, 25, 150, chunk=128)
    p, _, o, l = r.arrays()
    pw, _, ow, lw = w.arrays()

    def dec(pp, oo, ll, i):
        return "".join("ACGT"[(int(pp[oo[i] + k // 32]) >> (62 - 2 * (k % 32))) & 3]
                       for k in range(int(ll[i])))
    assert (lw == 150).all()
    for i in range(0, 300, 37):
        assert dec(pw, ow, lw, i) == dec(p, o, l, i)[25:175]
