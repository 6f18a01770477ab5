/*
 * align_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU alignment path, used as the
 * checker for the CUDA library.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load this file's shared object;
 * the product path (libgenomics_b200.so and the genomics_b200 package) never
 * calls into it.
 *
 * Every routine cites the reference function it restates (paths relative to
 * the reference project).  Arithmetic is int64_t throughout because Mojo's
 * `Int` is 64-bit.
 *
 * Pinning: the known-answer tests of tests/test_alignment.mojo:24-279,
 * tests/test_dna.mojo:86-120 and tests/test_sequence.mojo:30-83 are replayed
 * against these routines by tests/test_oracle_golden.py.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define OR_NEG_INF (-1000000LL) /* align_cpu.mojo:116, :406 */

static inline int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }
static inline int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

/* ------------------------------------------------------------------------ */
/* Encoding: genomics/core/dna.mojo, genomics/core/sequence.mojo             */
/* ------------------------------------------------------------------------ */

/* ascii_to_2bit (dna.mojo:25-40): ACGT/acgt -> 0..3, anything else -> 0xFF. */
int or_ascii_to_2bit(int c)
{
    switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 0xFF;
    }
}

/* get_base_from_word (dna.mojo:96-100): base `pos` of a word, MSB-first. */
static inline int64_t or_base_from_word(uint64_t w, int64_t pos)
{
    return (int64_t)((w >> (62 - 2 * pos)) & 3u);
}

/* SequenceView.get_base (sequence.mojo:96-101). */
static inline int64_t or_get_base(const uint64_t *words, int64_t pos)
{
    return or_base_from_word(words[pos / 32], pos % 32);
}

int64_t or_get_base_export(const uint64_t *words, int64_t pos)
{
    return or_get_base(words, pos);
}

/*
 * SequenceBatch.add_sequence (sequence.mojo:38-66) for one sequence:
 * writes ceil(len/32) packed words and as many NMask words.  Non-ACGT is
 * stored as A (0) and flagged LSB-first in the NMask (dna.mojo:107-141).
 * Returns the number of words written.
 */
int64_t or_pack_ascii(const uint8_t *src, int64_t len, uint64_t *packed,
                      uint64_t *nmask)
{
    int64_t n_words = (len + 31) / 32;
    for (int64_t w = 0; w < n_words; ++w) {
        int64_t base_off = w * 32;
        int64_t n = imin64(len - base_off, 32);
        uint64_t word = 0, nm = 0;
        for (int64_t i = 0; i < n; ++i) {
            int b = or_ascii_to_2bit(src[base_off + i]);
            if (b == 0xFF) {
                nm |= (uint64_t)1 << i;
                b = 0;
            }
            word |= (uint64_t)b << (62 - 2 * i);
        }
        packed[w] = word;
        if (nmask)
            nmask[w] = nm;
    }
    return n_words;
}

/* ------------------------------------------------------------------------ */
/* Banded Smith-Waterman: align_cpu.mojo:229-309                            */
/* ------------------------------------------------------------------------ */

/*
 * out[0..4] = score, query_start, ref_start, query_end, ref_end
 * (AlignResult, align_cpu.mojo:28-36; starts are always 0, :302-309).
 * A negative band gives an empty band (width <= 0) and the zero result.
 */
void or_sw_banded(const uint64_t *q, int64_t qlen, const uint64_t *r,
                  int64_t rlen, int64_t match, int64_t mismatch, int64_t go,
                  int64_t ge, int64_t band, int64_t *out)
{
    int64_t width = 2 * band + 1;
    int64_t best = 0, bq = 0, br = 0;
    if (width > 0) {
        int64_t *hp = (int64_t *)calloc((size_t)width, sizeof(int64_t));
        int64_t *hc = (int64_t *)calloc((size_t)width, sizeof(int64_t));
        int64_t *ec = (int64_t *)calloc((size_t)width, sizeof(int64_t));
        for (int64_t qi = 0; qi < qlen; ++qi) {
            /* rows restart from zero every query position (:261-263) */
            for (int64_t j = 0; j < width; ++j) {
                hc[j] = 0;
                ec[j] = 0;
            }
            int64_t qb = or_get_base(q, qi);
            for (int64_t off = 0; off < width; ++off) {
                int64_t ri = qi - band + off;
                if (ri < 0 || ri >= rlen)
                    continue; /* :265-268 */
                int64_t sub = (qb == or_get_base(r, ri)) ? match : mismatch;
                int64_t h_diag = hp[off];                         /* :277 */
                int64_t h_up = (off + 1 < width) ? hp[off + 1] : 0; /* :278 */
                int64_t h_left = (off > 0) ? hc[off - 1] : 0;       /* :279 */
                /* E extends from the left cell's E and opens from up (:282-283) */
                int64_t e_val = imax64(off > 0 ? ec[off - 1] + ge : -1000000LL,
                                       h_up + go + ge);
                /* F opens from the left H with no extension term (:287) */
                int64_t f_val = h_left + go + ge;
                int64_t cell = imax64(0, imax64(h_diag + sub, imax64(e_val, f_val)));
                hc[off] = cell;
                ec[off] = e_val;
                if (cell > best) { /* strict: first max in row-major order (:293-296) */
                    best = cell;
                    bq = qi;
                    br = ri;
                }
            }
            memcpy(hp, hc, (size_t)width * sizeof(int64_t)); /* :299-300 */
        }
        free(hp);
        free(hc);
        free(ec);
    }
    out[0] = best;
    out[1] = 0;
    out[2] = 0;
    out[3] = bq;
    out[4] = br;
}

/* ------------------------------------------------------------------------ */
/* Banded Needleman-Wunsch: align_cpu.mojo:312-377 (intended semantics)     */
/* ------------------------------------------------------------------------ */

/*
 * The reference creates H_prev/H_curr with capacity only and indexes them
 * without appending (align_cpu.mojo:327-337, :340-341).  This routine gives
 * both rows `width` elements, which is what the indexing assumes; every other
 * statement follows the reference.  out[] as for or_sw_banded, with
 * query_end = qlen-1 and ref_end = rlen-1 (:370-376).
 */
void or_nw_banded(const uint64_t *q, int64_t qlen, const uint64_t *r,
                  int64_t rlen, int64_t match, int64_t mismatch, int64_t go,
                  int64_t ge, int64_t band, int64_t *out)
{
    const int64_t NEG = -1000000LL; /* :325 */
    int64_t width = 2 * band + 1;
    int64_t final_score = NEG;
    if (width > 0) {
        int64_t *hp = (int64_t *)calloc((size_t)width, sizeof(int64_t));
        int64_t *hc = (int64_t *)calloc((size_t)width, sizeof(int64_t));
        for (int64_t j = 0; j < width; ++j) { /* :330-337 */
            int64_t ri = -band + j;
            if (ri < 0)
                hp[j] = NEG;
            else if (ri == 0)
                hp[j] = 0;
            else
                hp[j] = go + ri * ge;
        }
        for (int64_t qi = 0; qi < qlen; ++qi) {
            for (int64_t j = 0; j < width; ++j)
                hc[j] = NEG;
            int64_t qb = or_get_base(q, qi);
            for (int64_t off = 0; off < width; ++off) {
                int64_t ri = qi - band + off;
                if (ri < 0 || ri >= rlen)
                    continue;
                int64_t sub = (qb == or_get_base(r, ri)) ? match : mismatch;
                int64_t h_diag = hp[off];
                int64_t h_up = (off + 1 < width) ? hp[off + 1] : NEG;
                int64_t h_left = (off > 0) ? hc[off - 1] : NEG;
                int64_t cell = imax64(h_diag + sub,
                                      imax64(h_up + go + ge, h_left + go + ge));
                hc[off] = cell;
            }
            memcpy(hp, hc, (size_t)width * sizeof(int64_t));
        }
        int64_t final_off = (rlen - 1) - (qlen - 1) + band; /* :365-368 */
        if (final_off >= 0 && final_off < width)
            final_score = hp[final_off];
        free(hp);
        free(hc);
    }
    out[0] = final_score;
    out[1] = 0;
    out[2] = 0;
    out[3] = qlen - 1;
    out[4] = rlen - 1;
}

/* ------------------------------------------------------------------------ */
/* Gap-affine WFA, circular buffers: align_cpu.mojo:75-226 (as written)     */
/* ------------------------------------------------------------------------ */

/*
 * Statement-for-statement restatement, including the per-score reset of
 * all 2*max_err+1 diagonals (:153-156), the target-diagonal widening
 * (:158-162), the +-max_err clamp (:163-164) and unclamped offsets.
 * Returns the cost, or -1 when it exceeds max_err.  max_err < 0 is outside
 * the reference's domain (its buffers would have negative size) and
 * returns -2.
 */
int64_t or_wfa_affine(const uint64_t *q, int64_t qlen, const uint64_t *r,
                      int64_t rlen, int64_t x, int64_t o, int64_t e,
                      int64_t max_err)
{
    if (qlen == 0 && rlen == 0)
        return 0; /* :99-100 */
    if (max_err < 0)
        return -2;
    const int64_t NEG = OR_NEG_INF;
    int64_t n_diags = 2 * max_err + 1;
    int64_t doff = max_err;
    int64_t m_hist = imax64(x, o + e) + 1;
    int64_t ie_hist = e + 1;
    if (m_hist <= 0 || ie_hist <= 0)
        return -2;
    int64_t *M = (int64_t *)malloc((size_t)(m_hist * n_diags) * sizeof(int64_t));
    int64_t *I = (int64_t *)malloc((size_t)(ie_hist * n_diags) * sizeof(int64_t));
    int64_t *D = (int64_t *)malloc((size_t)(ie_hist * n_diags) * sizeof(int64_t));
    for (int64_t i = 0; i < m_hist * n_diags; ++i)
        M[i] = NEG;
    for (int64_t i = 0; i < ie_hist * n_diags; ++i) {
        I[i] = NEG;
        D[i] = NEG;
    }
    int64_t result = -1;
    M[doff] = 0; /* :130 */
    {
        int64_t row0 = M[doff], col0 = row0;
        while (row0 < qlen && col0 >= 0 && col0 < rlen) {
            if (or_get_base(q, row0) != or_get_base(r, col0))
                break;
            row0++;
            col0++;
        }
        M[doff] = row0; /* :140 */
    }
    int64_t target = qlen - rlen;
    if (target >= -max_err && target <= max_err) {
        if (M[doff + target] >= qlen) {
            result = 0;
            goto done;
        }
    }
    for (int64_t s = 1; s <= max_err; ++s) {
        int64_t ms = s % m_hist, is = s % ie_hist;
        for (int64_t j = 0; j < n_diags; ++j) { /* :153-156 */
            M[ms * n_diags + j] = NEG;
            I[is * n_diags + j] = NEG;
            D[is * n_diags + j] = NEG;
        }
        int64_t lo = imax64(-rlen, -s), hi = imin64(qlen, s);
        if (target < lo || target > hi) {
            lo = imin64(lo, target);
            hi = imax64(hi, target);
        }
        lo = imax64(lo, -max_err);
        hi = imin64(hi, max_err);
        for (int64_t d = lo; d <= hi; ++d) {
            int64_t di = d + doff;
            int64_t iv = NEG;
            if (di > 0) {
                if (s >= o + e) {
                    int64_t mv = M[((s - o - e) % m_hist) * n_diags + di - 1];
                    if (mv != NEG)
                        iv = imax64(iv, mv + 1);
                }
                if (s >= e) {
                    int64_t v = I[((s - e) % ie_hist) * n_diags + di - 1];
                    if (v != NEG)
                        iv = imax64(iv, v + 1);
                }
            }
            I[is * n_diags + di] = iv;
            int64_t dv = NEG;
            if (di < n_diags - 1) {
                if (s >= o + e) {
                    int64_t mv = M[((s - o - e) % m_hist) * n_diags + di + 1];
                    if (mv != NEG)
                        dv = imax64(dv, mv);
                }
                if (s >= e) {
                    int64_t v = D[((s - e) % ie_hist) * n_diags + di + 1];
                    if (v != NEG)
                        dv = imax64(dv, v);
                }
            }
            D[is * n_diags + di] = dv;
            int64_t mval = NEG;
            if (s >= x) {
                int64_t mv = M[((s - x) % m_hist) * n_diags + di];
                if (mv != NEG)
                    mval = imax64(mval, mv + 1);
            }
            if (iv != NEG)
                mval = imax64(mval, iv);
            if (dv != NEG)
                mval = imax64(mval, dv);
            M[ms * n_diags + di] = mval;
        }
        for (int64_t d = lo; d <= hi; ++d) { /* extend, :208-219 */
            int64_t di = d + doff;
            int64_t row = M[ms * n_diags + di];
            if (row == NEG || row < 0)
                continue;
            int64_t col = row - d;
            while (row < qlen && col >= 0 && col < rlen) {
                if (or_get_base(q, row) != or_get_base(r, col))
                    break;
                row++;
                col++;
            }
            M[ms * n_diags + di] = row;
        }
        if (target >= lo && target <= hi) { /* :222-224 */
            if (M[ms * n_diags + doff + target] >= qlen) {
                result = s;
                goto done;
            }
        }
    }
done:
    free(M);
    free(I);
    free(D);
    return result;
}

/* ------------------------------------------------------------------------ */
/* The same function computed over the live wavefront envelope only          */
/* ------------------------------------------------------------------------ */

/*
 * Returns exactly what or_wfa_affine returns, for x >= 1, e >= 1, o >= 0.
 * Each ring slot remembers the diagonal interval it wrote; reads outside it
 * are NEG, which is what the reference's full reset makes them.  Diagonals
 * inside [lo,hi] but outside the union of the sources' intervals would only
 * ever be assigned NEG, so they are not visited.  Work counters (may be NULL):
 * work[0] = wavefront cells visited, work[1] = bases consumed by extension,
 * work[2] = scores visited.
 */
int64_t or_wfa_affine_envelope(const uint64_t *q, int64_t qlen,
                               const uint64_t *r, int64_t rlen, int64_t x,
                               int64_t o, int64_t e, int64_t max_err,
                               int64_t *work)
{
    if (work)
        work[0] = work[1] = work[2] = 0;
    if (qlen == 0 && rlen == 0)
        return 0;
    if (max_err < 0 || x < 1 || e < 1 || o < 0)
        return -2;
    const int64_t NEG = OR_NEG_INF;
    int64_t m_hist = imax64(x, o + e) + 1, ie_hist = e + 1;
    /* diagonals can only lie in [max(-rlen,-max_err), min(qlen,max_err)] */
    int64_t kmin = imax64(-rlen, -max_err), kmax = imin64(qlen, max_err);
    int64_t target = qlen - rlen;
    if (kmin > 0)
        kmin = 0;
    if (kmax < 0)
        kmax = 0;
    int64_t width = kmax - kmin + 1;
    int64_t *M = (int64_t *)malloc((size_t)(m_hist * width) * sizeof(int64_t));
    int64_t *I = (int64_t *)malloc((size_t)(ie_hist * width) * sizeof(int64_t));
    int64_t *D = (int64_t *)malloc((size_t)(ie_hist * width) * sizeof(int64_t));
    int64_t *mlo = (int64_t *)malloc((size_t)m_hist * sizeof(int64_t));
    int64_t *mhi = (int64_t *)malloc((size_t)m_hist * sizeof(int64_t));
    int64_t *ilo = (int64_t *)malloc((size_t)ie_hist * sizeof(int64_t));
    int64_t *ihi = (int64_t *)malloc((size_t)ie_hist * sizeof(int64_t));
    int64_t *dlo = (int64_t *)malloc((size_t)ie_hist * sizeof(int64_t));
    int64_t *dhi = (int64_t *)malloc((size_t)ie_hist * sizeof(int64_t));
    for (int64_t i = 0; i < m_hist; ++i) {
        mlo[i] = 1;
        mhi[i] = 0; /* empty */
    }
    for (int64_t i = 0; i < ie_hist; ++i) {
        ilo[i] = dlo[i] = 1;
        ihi[i] = dhi[i] = 0;
    }
#define RD(buf, lo_, hi_, slot, k)                                           \
    (((k) >= lo_[slot] && (k) <= hi_[slot]) ? buf[(slot) * width + (k) - kmin] \
                                            : NEG)
    int64_t result = -1;
    {
        int64_t row0 = 0;
        while (row0 < qlen && row0 < rlen &&
               or_get_base(q, row0) == or_get_base(r, row0))
            row0++;
        if (work)
            work[1] += row0;
        M[0 * width + 0 - kmin] = row0;
        mlo[0] = 0;
        mhi[0] = 0;
        if (target >= -max_err && target <= max_err && target == 0 &&
            row0 >= qlen) {
            result = 0;
            goto done;
        }
    }
    for (int64_t s = 1; s <= max_err; ++s) {
        int64_t ms = s % m_hist, is = s % ie_hist;
        int64_t lo = imax64(-rlen, -s), hi = imin64(qlen, s);
        if (target < lo || target > hi) {
            lo = imin64(lo, target);
            hi = imax64(hi, target);
        }
        lo = imax64(lo, -max_err);
        hi = imin64(hi, max_err);
        /* union of the source intervals, shifted to the diagonals they feed */
        int64_t ulo = INT64_MAX, uhi = INT64_MIN;
        if (s >= x) {
            int64_t sl = (s - x) % m_hist;
            if (mlo[sl] <= mhi[sl]) {
                ulo = imin64(ulo, mlo[sl]);
                uhi = imax64(uhi, mhi[sl]);
            }
        }
        if (s >= o + e) {
            int64_t sl = (s - o - e) % m_hist;
            if (mlo[sl] <= mhi[sl]) {
                ulo = imin64(ulo, mlo[sl] - 1);
                uhi = imax64(uhi, mhi[sl] + 1);
            }
        }
        if (s >= e) {
            int64_t sl = (s - e) % ie_hist;
            if (ilo[sl] <= ihi[sl]) {
                ulo = imin64(ulo, ilo[sl] + 1);
                uhi = imax64(uhi, ihi[sl] + 1);
            }
            if (dlo[sl] <= dhi[sl]) {
                ulo = imin64(ulo, dlo[sl] - 1);
                uhi = imax64(uhi, dhi[sl] - 1);
            }
        }
        int64_t a = imax64(lo, ulo), b = imin64(hi, uhi);
        if (a > b) {
            mlo[ms] = ilo[is] = dlo[is] = 1;
            mhi[ms] = ihi[is] = dhi[is] = 0;
            continue; /* empty score: nothing can terminate here */
        }
        if (work) {
            work[0] += b - a + 1;
            work[2] += 1;
        }
        int64_t sm_x = (s - x) % m_hist, sm_oe = (s - o - e) % m_hist;
        int64_t se = (s >= e) ? (s - e) % ie_hist : -1;
        /* I and D of score s only read score s-e < s, so every value below is
           read from slots written before this score started. */
        for (int64_t d = a; d <= b; ++d) {
            int64_t iv = NEG, dv = NEG, mval = NEG, v;
            if (s >= o + e) {
                v = RD(M, mlo, mhi, sm_oe, d - 1);
                if (v != NEG)
                    iv = imax64(iv, v + 1);
                v = RD(M, mlo, mhi, sm_oe, d + 1);
                if (v != NEG)
                    dv = imax64(dv, v);
            }
            if (se >= 0) {
                v = RD(I, ilo, ihi, se, d - 1);
                if (v != NEG)
                    iv = imax64(iv, v + 1);
                v = RD(D, dlo, dhi, se, d + 1);
                if (v != NEG)
                    dv = imax64(dv, v);
            }
            if (s >= x) {
                v = RD(M, mlo, mhi, sm_x, d);
                if (v != NEG)
                    mval = imax64(mval, v + 1);
            }
            if (iv != NEG)
                mval = imax64(mval, iv);
            if (dv != NEG)
                mval = imax64(mval, dv);
            I[is * width + d - kmin] = iv;
            D[is * width + d - kmin] = dv;
            M[ms * width + d - kmin] = mval;
        }
        ilo[is] = dlo[is] = mlo[ms] = a;
        ihi[is] = dhi[is] = mhi[ms] = b;
        for (int64_t d = a; d <= b; ++d) {
            int64_t row = M[ms * width + d - kmin];
            if (row == NEG || row < 0)
                continue;
            int64_t col = row - d, row_in = row;
            while (row < qlen && col >= 0 && col < rlen &&
                   or_get_base(q, row) == or_get_base(r, col)) {
                row++;
                col++;
            }
            if (work)
                work[1] += row - row_in;
            M[ms * width + d - kmin] = row;
        }
        if (target >= lo && target <= hi && target >= a && target <= b) {
            if (M[ms * width + target - kmin] >= qlen) {
                result = s;
                goto done;
            }
        }
    }
done:
#undef RD
    free(M);
    free(I);
    free(D);
    free(mlo);
    free(mhi);
    free(ilo);
    free(ihi);
    free(dlo);
    free(dhi);
    return result;
}

/* ------------------------------------------------------------------------ */
/* Gap-affine WFA with full history and CIGAR: align_cpu.mojo:380-623       */
/* ------------------------------------------------------------------------ */

/*
 * Writes the run-length extended CIGAR ("3=1X2I") into cigar (NUL
 * terminated, at most cap bytes including the NUL) and returns the cost,
 * -1 past max_err (empty CIGAR), or -3 when cap is too small.
 */
int64_t or_wfa_cigar(const uint64_t *q, int64_t qlen, const uint64_t *r,
                     int64_t rlen, int64_t x, int64_t o, int64_t e,
                     int64_t max_err, char *cigar, int64_t cap)
{
    if (cap < 1)
        return -3;
    cigar[0] = 0;
    if (qlen == 0 && rlen == 0)
        return 0; /* :396-397 */
    if (max_err < 0)
        return -2;
    const int64_t NEG = OR_NEG_INF;
    int64_t n_diags = 2 * max_err + 1, off = max_err;
    int64_t total = (max_err + 1) * n_diags;
    int64_t *Mpre = (int64_t *)malloc((size_t)total * sizeof(int64_t));
    int64_t *Mfull = (int64_t *)malloc((size_t)total * sizeof(int64_t));
    int64_t *Ia = (int64_t *)malloc((size_t)total * sizeof(int64_t));
    int64_t *Da = (int64_t *)malloc((size_t)total * sizeof(int64_t));
    for (int64_t i = 0; i < total; ++i)
        Mpre[i] = Mfull[i] = Ia[i] = Da[i] = NEG;
    Mpre[off] = 0; /* :423-427 */
    int64_t r0 = 0;
    while (r0 < qlen && r0 < rlen && or_get_base(q, r0) == or_get_base(r, r0))
        r0++;
    Mfull[off] = r0;
    int64_t target = qlen - rlen, opt = -1;
    if (target >= -max_err && target <= max_err && Mfull[off + target] >= qlen)
        opt = 0;
    if (opt == -1) {
        for (int64_t s = 1; s <= max_err; ++s) { /* :438-504 */
            int64_t lo = imax64(-rlen, -s), hi = imin64(qlen, s);
            if (target < lo)
                lo = imin64(lo, target);
            if (target > hi)
                hi = imax64(hi, target);
            lo = imax64(lo, -max_err);
            hi = imin64(hi, max_err);
            for (int64_t d = lo; d <= hi; ++d) {
                int64_t di = d + off;
                int64_t iv = NEG;
                if (di > 0) {
                    if (s >= o + e) {
                        int64_t mv = Mfull[(s - o - e) * n_diags + di - 1];
                        if (mv != NEG)
                            iv = imax64(iv, mv + 1);
                    }
                    if (s >= e) {
                        int64_t v = Ia[(s - e) * n_diags + di - 1];
                        if (v != NEG)
                            iv = imax64(iv, v + 1);
                    }
                }
                Ia[s * n_diags + di] = iv;
                int64_t dv = NEG;
                if (di < n_diags - 1) {
                    if (s >= o + e) {
                        int64_t mv = Mfull[(s - o - e) * n_diags + di + 1];
                        if (mv != NEG)
                            dv = imax64(dv, mv);
                    }
                    if (s >= e) {
                        int64_t v = Da[(s - e) * n_diags + di + 1];
                        if (v != NEG)
                            dv = imax64(dv, v);
                    }
                }
                Da[s * n_diags + di] = dv;
                int64_t mval = NEG;
                if (s >= x) {
                    int64_t mv = Mfull[(s - x) * n_diags + di];
                    if (mv != NEG)
                        mval = imax64(mval, mv + 1);
                }
                if (iv != NEG)
                    mval = imax64(mval, iv);
                if (dv != NEG)
                    mval = imax64(mval, dv);
                Mpre[s * n_diags + di] = mval;
                if (mval != NEG) { /* extend in place, :489-498 */
                    int64_t row = mval, col = row - d;
                    while (row < qlen && col >= 0 && col < rlen) {
                        if (or_get_base(q, row) != or_get_base(r, col))
                            break;
                        row++;
                        col++;
                    }
                    Mfull[s * n_diags + di] = row;
                }
            }
            if (target >= lo && target <= hi &&
                Mfull[s * n_diags + off + target] >= qlen) {
                opt = s;
                break;
            }
        }
    }
    int64_t ret = opt;
    if (opt == -1)
        goto out;
    {
        /* backtrace (:509-601); ops: 0 '=', 1 'X', 2 'I', 3 'D' */
        int64_t ops_cap = 2 * (qlen + rlen) + 16, n_ops = 0;
        uint8_t *ops = (uint8_t *)malloc((size_t)ops_cap);
        int64_t cs = opt, cd = target, cm = 0;
        int64_t crow = Mfull[opt * n_diags + target + off];
        for (;;) {
            int64_t di = cd + off;
            if (n_ops + (cm == 0 ? crow + 2 : 2) > ops_cap) {
                ops_cap = 2 * ops_cap + crow + 2;
                ops = (uint8_t *)realloc(ops, (size_t)ops_cap);
            }
            if (cm == 0) {
                int64_t pre = Mpre[cs * n_diags + di];
                for (int64_t t = 0; t < crow - pre; ++t)
                    ops[n_ops++] = 0;
                crow = pre;
                if (cs == 0 && cd == 0)
                    break;
                if (cs >= x) {
                    int64_t pm = Mfull[(cs - x) * n_diags + di];
                    if (pm != NEG && pm + 1 == crow) {
                        ops[n_ops++] = 1;
                        cs -= x;
                        crow = pm;
                        continue;
                    }
                }
                int64_t ih = Ia[cs * n_diags + di];
                if (ih != NEG && ih == crow) {
                    cm = 1;
                    continue;
                }
                int64_t dh = Da[cs * n_diags + di];
                if (dh != NEG && dh == crow) {
                    cm = 2;
                    continue;
                }
                break;
            } else if (cm == 1) {
                ops[n_ops++] = 2;
                int64_t pd = cd - 1, pdi = pd + off;
                if (cs >= o + e && pdi >= 0) {
                    int64_t mv = Mfull[(cs - o - e) * n_diags + pdi];
                    if (mv != NEG && mv + 1 == crow) {
                        cs -= o + e;
                        cd = pd;
                        crow = mv;
                        cm = 0;
                        continue;
                    }
                }
                if (cs >= e && pdi >= 0) {
                    int64_t iv = Ia[(cs - e) * n_diags + pdi];
                    if (iv != NEG && iv + 1 == crow) {
                        cs -= e;
                        cd = pd;
                        crow = iv;
                        cm = 1;
                        continue;
                    }
                }
                break;
            } else {
                ops[n_ops++] = 3;
                int64_t pd = cd + 1, pdi = pd + off;
                if (cs >= o + e && pdi < n_diags) {
                    int64_t mv = Mfull[(cs - o - e) * n_diags + pdi];
                    if (mv != NEG && mv == crow) {
                        cs -= o + e;
                        cd = pd;
                        crow = mv;
                        cm = 0;
                        continue;
                    }
                }
                if (cs >= e && pdi < n_diags) {
                    int64_t dv = Da[(cs - e) * n_diags + pdi];
                    if (dv != NEG && dv == crow) {
                        cs -= e;
                        cd = pd;
                        crow = dv;
                        cm = 2;
                        continue;
                    }
                }
                break;
            }
        }
        /* run-length encode, reading ops back to front (:603-621) */
        static const char opc[4] = {'=', 'X', 'I', 'D'};
        int64_t pos = 0;
        int64_t i = n_ops - 1;
        while (i >= 0) {
            uint8_t op = ops[i];
            int64_t cnt = 1;
            while (i - cnt >= 0 && ops[i - cnt] == op)
                cnt++;
            char buf[32];
            int len = 0;
            int64_t c = cnt;
            char tmp[24];
            int tl = 0;
            do {
                tmp[tl++] = (char)('0' + c % 10);
                c /= 10;
            } while (c > 0);
            while (tl > 0)
                buf[len++] = tmp[--tl];
            buf[len++] = opc[op];
            if (pos + len + 1 > cap) {
                free(ops);
                cigar[0] = 0;
                ret = -3;
                goto out;
            }
            memcpy(cigar + pos, buf, (size_t)len);
            pos += len;
            i -= cnt;
        }
        cigar[pos] = 0;
        free(ops);
    }
out:
    free(Mpre);
    free(Mfull);
    free(Ia);
    free(Da);
    return ret;
}

/* ------------------------------------------------------------------------ */
/* Multithreaded batch drivers over SequenceBatch-shaped arrays             */
/* ------------------------------------------------------------------------ */

/*
 * Pair i is (query i, ref i), as in launch_banded_sw / launch_wfa_affine
 * (genomics/gpu/align_gpu.mojo:460-535).  Per-sequence word offsets and
 * lengths follow SequenceBatch (genomics/core/sequence.mojo:23-36).  The
 * optional per-pair band array overrides `band` (mixed-band batches).
 */
typedef struct {
    const uint64_t *qp, *rp;
    const int64_t *qoff, *qlen, *roff, *rlen, *bands;
    int64_t n;
    int64_t p0, p1, p2, p3, p4; /* scoring parameters */
    int kind;                   /* 0 sw, 1 wfa, 2 wfa envelope, 3 nw */
    int32_t *o0, *o1, *o2;
    int64_t *work;              /* per-thread work accumulators (3 each) */
    int tid, nthreads;
} or_job;

static void *or_worker(void *arg)
{
    or_job *j = (or_job *)arg;
    int64_t w[3] = {0, 0, 0};
    for (int64_t i = j->tid; i < j->n; i += j->nthreads) {
        const uint64_t *q = j->qp + j->qoff[i];
        const uint64_t *r = j->rp + j->roff[i];
        if (j->kind == 0 || j->kind == 3) {
            int64_t out[5];
            int64_t band = j->bands ? j->bands[i] : j->p4;
            if (j->kind == 0)
                or_sw_banded(q, j->qlen[i], r, j->rlen[i], j->p0, j->p1, j->p2,
                             j->p3, band, out);
            else
                or_nw_banded(q, j->qlen[i], r, j->rlen[i], j->p0, j->p1, j->p2,
                             j->p3, band, out);
            j->o0[i] = (int32_t)out[0];
            j->o1[i] = (int32_t)out[3];
            j->o2[i] = (int32_t)out[4];
        } else if (j->kind == 1) {
            j->o0[i] = (int32_t)or_wfa_affine(q, j->qlen[i], r, j->rlen[i],
                                              j->p0, j->p1, j->p2, j->p3);
        } else {
            int64_t ww[3];
            j->o0[i] = (int32_t)or_wfa_affine_envelope(
                q, j->qlen[i], r, j->rlen[i], j->p0, j->p1, j->p2, j->p3, ww);
            w[0] += ww[0];
            w[1] += ww[1];
            w[2] += ww[2];
        }
    }
    if (j->work) {
        j->work[3 * j->tid + 0] = w[0];
        j->work[3 * j->tid + 1] = w[1];
        j->work[3 * j->tid + 2] = w[2];
    }
    return NULL;
}

static void or_run(or_job *base, int nthreads)
{
    if (nthreads < 1)
        nthreads = 1;
    if (nthreads > 256)
        nthreads = 256;
    pthread_t th[256];
    or_job jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = *base;
        jobs[t].tid = t;
        jobs[t].nthreads = nthreads;
    }
    for (int t = 1; t < nthreads; ++t)
        pthread_create(&th[t], NULL, or_worker, &jobs[t]);
    or_worker(&jobs[0]);
    for (int t = 1; t < nthreads; ++t)
        pthread_join(th[t], NULL);
}

/* SW batch: out_score/out_qend/out_rend per pair. */
void or_sw_batch(const uint64_t *qp, const int64_t *qoff, const int64_t *qlen,
                 const uint64_t *rp, const int64_t *roff, const int64_t *rlen,
                 int64_t n, int64_t match, int64_t mismatch, int64_t go,
                 int64_t ge, int64_t band, const int64_t *bands,
                 int32_t *out_score, int32_t *out_qend, int32_t *out_rend,
                 int nthreads)
{
    or_job j;
    memset(&j, 0, sizeof j);
    j.qp = qp; j.rp = rp; j.qoff = qoff; j.qlen = qlen; j.roff = roff;
    j.rlen = rlen; j.bands = bands; j.n = n;
    j.p0 = match; j.p1 = mismatch; j.p2 = go; j.p3 = ge; j.p4 = band;
    j.kind = 0;
    j.o0 = out_score; j.o1 = out_qend; j.o2 = out_rend;
    or_run(&j, nthreads);
}

/* NW batch (intended semantics, see or_nw_banded). */
void or_nw_batch(const uint64_t *qp, const int64_t *qoff, const int64_t *qlen,
                 const uint64_t *rp, const int64_t *roff, const int64_t *rlen,
                 int64_t n, int64_t match, int64_t mismatch, int64_t go,
                 int64_t ge, int64_t band, const int64_t *bands,
                 int32_t *out_score, int nthreads)
{
    int32_t *tmp = (int32_t *)malloc((size_t)(2 * (n > 0 ? n : 1)) * sizeof(int32_t));
    or_job j;
    memset(&j, 0, sizeof j);
    j.qp = qp; j.rp = rp; j.qoff = qoff; j.qlen = qlen; j.roff = roff;
    j.rlen = rlen; j.bands = bands; j.n = n;
    j.p0 = match; j.p1 = mismatch; j.p2 = go; j.p3 = ge; j.p4 = band;
    j.kind = 3;
    j.o0 = out_score; j.o1 = tmp; j.o2 = tmp + (n > 0 ? n : 1);
    or_run(&j, nthreads);
    free(tmp);
}

/*
 * WFA batch.  envelope=0 runs the statement-for-statement routine,
 * envelope=1 the live-envelope one (same results, far less work for large
 * max_err); work (3 int64, may be NULL) sums the envelope work counters.
 */
void or_wfa_batch(const uint64_t *qp, const int64_t *qoff, const int64_t *qlen,
                  const uint64_t *rp, const int64_t *roff, const int64_t *rlen,
                  int64_t n, int64_t x, int64_t o, int64_t e, int64_t max_err,
                  int envelope, int32_t *out_cost, int64_t *work, int nthreads)
{
    if (nthreads < 1)
        nthreads = 1;
    if (nthreads > 256)
        nthreads = 256;
    int64_t *w = (int64_t *)calloc((size_t)(3 * nthreads), sizeof(int64_t));
    or_job j;
    memset(&j, 0, sizeof j);
    j.qp = qp; j.rp = rp; j.qoff = qoff; j.qlen = qlen; j.roff = roff;
    j.rlen = rlen; j.n = n;
    j.p0 = x; j.p1 = o; j.p2 = e; j.p3 = max_err;
    j.kind = envelope ? 2 : 1;
    j.o0 = out_cost;
    j.work = w;
    or_run(&j, nthreads);
    if (work) {
        work[0] = work[1] = work[2] = 0;
        for (int t = 0; t < nthreads; ++t) {
            work[0] += w[3 * t];
            work[1] += w[3 * t + 1];
            work[2] += w[3 * t + 2];
        }
    }
    free(w);
}
