"""The oracle pinned against the reference's own known answers, and against an
independent small restatement.  CPU only."""
import random

import numpy as np
import pytest

# default_config (genomics/cpu/align_cpu.mojo:46-53)
DEF = dict(match=2, mismatch=-3, gap_open=-5, gap_extend=-2)


def test_sw_known_answers(oracle, known):
    for case in known["sw"]:
        s = oracle.sw_banded(case["q"], case["r"], band=case["band"], **DEF)
        if "score" in case:
            assert s[0] == case["score"], case["src"]
        else:
            assert s[0] >= case["score_at_least"] and s[0] > 0, case["src"]
        assert s[1] == 0 and s[2] == 0


def test_nw_known_answers(oracle, known):
    for case in known["nw"]:
        s = oracle.nw_banded(case["q"], case["r"], band=case["band"], **DEF)
        assert s[0] == case["score"], case["src"]


def test_wfa_known_answers(oracle, known):
    for case in known["wfa"]:
        assert oracle.wfa_affine(case["q"], case["r"]) == case["cost"], case["src"]
        assert oracle.wfa_affine(case["q"], case["r"], envelope=True) == case["cost"], case["src"]


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


def test_wfa_cigar_known_answers(oracle, known):
    for case in known["wfa_cigar"]:
        cost, cig = oracle.wfa_cigar(case["q"], case["r"])
        assert cost == case["cost"] and cig == case["cigar"], case["src"]
    for q, r in known["wfa_cigar_consistency"]["pairs"]:
        cost, cig = oracle.wfa_cigar(q, r)
        assert cost == oracle.wfa_affine(q, r)
        assert _cigar_cost(cig, 4, 6, 2) == cost
        assert _cigar_len(cig, "=XI") == len(q)
        assert _cigar_len(cig, "=XD") == len(r)


def _cigar_walk_ok(cigar, q, r):
    """'=' runs pair equal bases, 'X' runs unequal ones, I consumes the query, D the
    reference, and the walk ends at both ends."""
    i = j = cnt = 0
    for ch in cigar:
        if ch.isdigit():
            cnt = cnt * 10 + int(ch)
            continue
        for _ in range(cnt):
            if ch in "=X":
                if i >= len(q) or j >= len(r) or (q[i] == r[j]) != (ch == "="):
                    return False
                i += 1
                j += 1
            elif ch == "I":
                i += 1
            else:
                j += 1
        cnt = 0
    return i == len(q) and j == len(r)


def test_wfa_cigar_properties_on_random_pairs(oracle):
    """For random pairs and penalties: the CIGAR's cost equals the cost, which equals
    wfa_affine's; the CIGAR walks both sequences with '=' on equal and 'X' on unequal
    bases; past max_error the cost is -1 and the CIGAR empty."""
    rng = random.Random(380)
    for _ in range(300):
        q = _rand_seq(rng, rng.randint(0, 120))
        r = list(q)
        for _k in range(rng.randint(0, 12)):
            op, pos = rng.random(), rng.randint(0, max(len(r) - 1, 0))
            if op < 0.5 and r:
                r[pos] = rng.choice("ACGT")
            elif op < 0.75:
                r.insert(pos, rng.choice("ACGT"))
            elif r:
                del r[pos]
        r = "".join(r) if rng.random() < 0.9 else _rand_seq(rng, rng.randint(0, 60))
        x, o, e = rng.randint(1, 6), rng.randint(0, 8), rng.randint(1, 4)
        me = rng.choice([10, 60, 300])
        cost, cig = oracle.wfa_cigar(q, r, x, o, e, me)
        assert cost == oracle.wfa_affine(q, r, x, o, e, me)
        if cost < 0:
            assert cig == ""
            continue
        assert _cigar_cost(cig, x, o, e) == cost, (q, r, x, o, e, cig)
        assert _cigar_walk_ok(cig, q, r), (q, r, cig)


def test_encoding_known_answers(oracle, known):
    enc = known["encoding"]
    for c, v in enc["ascii_to_2bit"]["cases"]:
        assert oracle.lib().or_ascii_to_2bit(c) == v
    w = np.array([int(enc["get_base_from_word"]["word_hex"], 16)], np.uint64)
    for i, b in enumerate(enc["get_base_from_word"]["bases"]):
        assert oracle.lib().or_get_base_export(oracle._p(w, oracle._u64p), i) == b
    p, m = oracle.pack(enc["view_33"]["seq"])
    assert p.size == enc["view_33"]["word_count"]
    assert int(p[1] >> np.uint64(62)) == enc["view_33"]["last_base"]
    p, m = oracle.pack(enc["n_tracking"]["seq"])
    assert [bool((int(m[0]) >> i) & 1) for i in range(4)] == enc["n_tracking"]["is_n"]


# ---- an independent, deliberately naive restatement for small cases ----------------

def _base(s, i):
    return {"A": 0, "C": 1, "G": 2, "T": 3}.get(s[i].upper(), 0)


def _sw_naive(q, r, m, mm, go, ge, b):
    """Band cell (qi, j), ri = qi - b + j; dictionaries default to 0 for
    skipped cells, which is what align_cpu.mojo:261-263 resets them to."""
    H, E = {}, {}
    best = (0, 0, 0)
    for qi in range(len(q)):
        for j in range(2 * b + 1):
            ri = qi - b + j
            if ri < 0 or ri >= len(r):
                continue
            sub = m if _base(q, qi) == _base(r, ri) else mm
            hd = H.get((qi - 1, j), 0)
            hu = H.get((qi - 1, j + 1), 0) if j + 1 <= 2 * b else 0
            hl = H.get((qi, j - 1), 0) if j > 0 else 0
            el = E.get((qi, j - 1), 0) + ge if j > 0 else -1000000
            e = max(el, hu + go + ge)
            f = hl + go + ge
            h = max(0, hd + sub, e, f)
            H[(qi, j)] = h
            E[(qi, j)] = e
            if h > best[0]:
                best = (h, qi, ri)
    return best


def _rand_seq(rng, n, alphabet="ACGT"):
    return "".join(rng.choice(alphabet) for _ in range(n))


def test_sw_matches_naive_restatement(oracle):
    rng = random.Random(7)
    for _ in range(300):
        q = _rand_seq(rng, rng.randint(0, 40), "ACGTN")
        r = _rand_seq(rng, rng.randint(0, 40), "ACGTN")
        if rng.random() < 0.5 and q:
            r = q[: rng.randint(0, len(q))] + _rand_seq(rng, rng.randint(0, 8))
        b = rng.randint(0, 12)
        prm = (rng.randint(0, 4), -rng.randint(0, 5), -rng.randint(0, 6), -rng.randint(0, 3))
        if rng.random() < 0.1:  # configurations outside the usual signs
            prm = (rng.randint(-2, 4), rng.randint(-5, 3), rng.randint(-6, 3), rng.randint(-3, 2))
        got = oracle.sw_banded(q, r, *prm, band=b)
        s, qi, ri = _sw_naive(q, r, *prm, b)
        assert (got[0], got[3], got[4]) == (s, qi, ri), (q, r, prm, b)


def _nw_naive(q, r, m, mm, go, ge, b):
    """Banded NW in (row, reference position) coordinates, the oracle's intended
    semantics of align_cpu.mojo:312-377 written without band offsets: row 0 reads
    the initial band row (indexed like row 0, :330-337), later rows the previous
    row's cells; skipped and out-of-band cells are NEG; the end cell is
    (qlen - 1, rlen - 1) when it lies in the band (:365-368)."""
    NEG = -1000000
    qn, rn = len(q), len(r)

    def init(x):  # the initial band row at reference position x
        return NEG if x < 0 else (0 if x == 0 else go + x * ge)

    H = {}
    for qi in range(qn):
        for ri in range(max(0, qi - b), min(rn, qi + b + 1)):
            sub = m if _base(q, qi) == _base(r, ri) else mm
            if qi == 0:
                hd = init(ri)
                hu = init(ri + 1) if ri + 1 <= b else NEG
            else:
                hd = H.get((qi - 1, ri - 1), NEG) if ri - 1 >= qi - 1 - b else NEG
                hu = H.get((qi - 1, ri), NEG) if ri <= qi - 1 + b else NEG
            hl = H.get((qi, ri - 1), NEG) if ri - 1 >= qi - b else NEG
            H[(qi, ri)] = max(hd + sub, hu + go + ge, hl + go + ge)
    if qn == 0:  # no row ran: the end cell reads the initial row at offset rlen - 1 + b + 1
        off = (rn - 1) - (0 - 1) + b
        return init(off - b) if 0 <= off < 2 * b + 1 else NEG
    if abs((rn - 1) - (qn - 1)) > b:
        return NEG
    return H.get((qn - 1, rn - 1), NEG)


def test_nw_matches_naive_restatement(oracle):
    rng = random.Random(13)
    for _ in range(400):
        q = _rand_seq(rng, rng.randint(0, 40), "ACGTN")
        r = _rand_seq(rng, rng.randint(0, 40), "ACGTN")
        if rng.random() < 0.5 and q:
            r = q[: rng.randint(0, len(q))] + _rand_seq(rng, rng.randint(0, 8))
        b = rng.randint(0, 12)
        prm = (rng.randint(0, 4), -rng.randint(0, 5), -rng.randint(0, 6), -rng.randint(0, 3))
        got = oracle.nw_banded(q, r, *prm, band=b)
        assert got[0] == _nw_naive(q, r, *prm, b), (q, r, prm, b)


def test_wfa_envelope_equals_statement_for_statement(oracle):
    rng = random.Random(11)
    for _ in range(400):
        q = _rand_seq(rng, rng.randint(0, 60))
        if rng.random() < 0.7 and q:
            r = list(q)
            for _k in range(rng.randint(0, 8)):
                op = rng.random()
                pos = rng.randint(0, max(len(r) - 1, 0))
                if op < 0.5 and r:
                    r[pos] = rng.choice("ACGT")
                elif op < 0.75:
                    r.insert(pos, rng.choice("ACGT"))
                elif r:
                    del r[pos]
            r = "".join(r)
        else:
            r = _rand_seq(rng, rng.randint(0, 60))
        x, o, e = rng.randint(1, 6), rng.randint(0, 8), rng.randint(1, 4)
        me = rng.choice([0, 1, 5, 20, 60, 200])
        a = oracle.wfa_affine(q, r, x, o, e, me)
        b = oracle.wfa_affine(q, r, x, o, e, me, envelope=True)
        assert a == b, (q, r, x, o, e, me)


def test_wfa_envelope_equals_statement_for_statement_long(oracle):
    """Pairs of 300-3,000 bases at 1-10% divergence: the live-envelope form (what the
    long-pair parity checks use) equals the statement-for-statement form at the exact
    cost, one below it (-1) and above it."""
    rng = random.Random(1500)
    for _ in range(60):
        q = _rand_seq(rng, rng.randint(300, 3000))
        r = list(q)
        for _k in range(int(len(q) * rng.uniform(0.01, 0.10))):
            op = rng.random()
            pos = rng.randint(0, len(r) - 1)
            if op < 0.7:
                r[pos] = rng.choice("ACGT")
            elif op < 0.85:
                r.insert(pos, rng.choice("ACGT"))
            elif len(r) > 1:
                del r[pos]
        r = "".join(r)
        x, o, e = rng.choice([(4, 6, 2), (1, 1, 1), (3, 5, 1), (6, 8, 3), (2, 0, 2)])
        cost = oracle.wfa_affine(q, r, x, o, e, 4 * (len(q) + len(r)), envelope=True)
        assert cost >= 0
        for me in (cost, cost - 1, cost + 17):
            if me < 0:
                continue
            a = oracle.wfa_affine(q, r, x, o, e, me)
            b = oracle.wfa_affine(q, r, x, o, e, me, envelope=True)
            assert a == b == (cost if me >= cost else -1), (len(q), len(r), x, o, e, me, a, b)


def test_wfa_batch_driver_matches_single(oracle):
    from genomics_b200 import synth
    q, r, _, _ = synth.generate(2, 40, seed=5)
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    env, work = oracle.wfa_batch(qp, qo, ql, rp, ro, rl, 4, 6, 2, me, envelope=True, threads=4)
    assert (env >= 0).all() and work[0] > 0
    # the statement-for-statement routine on the shortest pairs
    for i in np.argsort(ql)[:8]:
        w = oracle.lib().or_wfa_affine(oracle._p(qp[qo[i]:], oracle._u64p), int(ql[i]),
                                       oracle._p(rp[ro[i]:], oracle._u64p), int(rl[i]), 4, 6, 2, me)
        assert w == env[i]
