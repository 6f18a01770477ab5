/*
 * synth.c -- seeded synthetic pair generator for the alignment workloads.
 *
 * The reference benchmarks on no public dataset (its own harness draws LCG
 * random DNA, benchmarks/harness.mojo:59-66), so every workload here is
 * generated from a seed.  Output is already in SequenceBatch layout
 * (genomics/core/sequence.mojo:23-36): 2-bit MSB-first packed words, one
 * NMask word per packed word (LSB-first), per-sequence word offsets and base
 * lengths.  Non-ACGT positions (the N runs of the mixed workload) are stored
 * as A and flagged in the NMask, exactly as add_sequence does
 * (sequence.mojo:53-57).
 *
 * Random numbers: SplitMix64 seeds xoshiro256** (Blackman & Vigna).
 *
 * Workloads (id):
 *   0/1  reads: a uniform 1 Mbp (0) or 10 Mbp (1) reference; the target is
 *        the 200 bp window [origin-25, origin+175); the query walks the
 *        reference from origin with 2% substitutions and 0.5% indel events
 *        (ins/del 50/50, length geometric mean 2) until it holds 150 bases.
 *   2    WFA pairs: L = round(exp(U(ln 100, ln 10000))); the query is
 *        uniform random, the reference is the query mutated at divergence
 *        d ~ U(1%,10%) (70% substitutions, 30% indels, length geometric mean 3).
 *   3    mixed SW: q ~ U{100..2000}; target = a random 10 Mbp-reference window
 *        of round(1.25 q) bases; query = mutated walk from the window start,
 *        d ~ U(1%,8%), until q bases; band from {16,32,64,128}; N runs
 *        (start probability 0.001 per base, length geometric mean 10) in both.
 *   4    serving pool: each pair is SW (band 32/64/128) or WFA with p = 0.5,
 *        L log-uniform 100..20000, d ~ U(0,15%), mutated like workload 2.
 *   100  the reference harness's own input: pair i is make_random_batch's
 *        sequence i against itself (harness.mojo:59-66), fixed length.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t s[4];
} xs_t;

static uint64_t splitmix64(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t xs_next(xs_t *r)
{
    uint64_t *s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
}

static void xs_seed(xs_t *r, uint64_t seed)
{
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i)
        r->s[i] = splitmix64(&x);
}

static inline double xs_unif(xs_t *r) { return (double)(xs_next(r) >> 11) * 0x1.0p-53; }
static inline int64_t xs_int(xs_t *r, int64_t n) /* [0, n) */
{
    return (int64_t)(((__uint128_t)xs_next(r) * (uint64_t)n) >> 64);
}
static inline int64_t xs_geom(xs_t *r, double p) /* support 1,2,..., mean 1/p */
{
    int64_t k = 1;
    while (xs_unif(r) >= p)
        ++k;
    return k;
}

/* ---- growable ASCII buffer ------------------------------------------------ */
typedef struct {
    uint8_t *p;
    int64_t n, cap;
} buf_t;

static void bput(buf_t *b, uint8_t c)
{
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 4096;
        b->p = (uint8_t *)realloc(b->p, (size_t)b->cap);
    }
    b->p[b->n++] = c;
}

static const uint8_t ACGT[4] = {'A', 'C', 'G', 'T'};

/* ---- growable SequenceBatch ------------------------------------------------ */
typedef struct {
    uint64_t *packed, *nmask;
    int64_t *offsets, *lengths;
    int64_t count, n_words, cap_words, cap_seqs;
} sb_t;

static void sb_add(sb_t *b, const uint8_t *s, int64_t len)
{
    int64_t nw = (len + 31) / 32;
    if (b->n_words + nw > b->cap_words) {
        int64_t c = b->cap_words ? b->cap_words : 1024;
        while (c < b->n_words + nw)
            c *= 2;
        b->packed = (uint64_t *)realloc(b->packed, (size_t)c * 8);
        b->nmask = (uint64_t *)realloc(b->nmask, (size_t)c * 8);
        b->cap_words = c;
    }
    if (b->count == b->cap_seqs) {
        b->cap_seqs = b->cap_seqs ? 2 * b->cap_seqs : 1024;
        b->offsets = (int64_t *)realloc(b->offsets, (size_t)b->cap_seqs * 8);
        b->lengths = (int64_t *)realloc(b->lengths, (size_t)b->cap_seqs * 8);
    }
    for (int64_t w = 0; w < nw; ++w) {
        int64_t n = len - 32 * w;
        if (n > 32)
            n = 32;
        uint64_t word = 0, nm = 0;
        for (int64_t i = 0; i < n; ++i) {
            uint8_t c = s[32 * w + i];
            uint64_t code;
            switch (c) {
            case 'A': case 'a': code = 0; break;
            case 'C': case 'c': code = 1; break;
            case 'G': case 'g': code = 2; break;
            case 'T': case 't': code = 3; break;
            default: code = 0; nm |= 1ull << i; break;
            }
            word |= code << (62 - 2 * i);
        }
        b->packed[b->n_words + w] = word;
        b->nmask[b->n_words + w] = nm;
    }
    b->offsets[b->count] = b->n_words;
    b->lengths[b->count] = len;
    b->count++;
    b->n_words += nw;
}

/* Output handle returned to the caller (freed by gs_free). */
typedef struct {
    uint64_t *q_packed, *q_nmask;
    int64_t *q_offsets, *q_lengths;
    int64_t q_words;
    uint64_t *r_packed, *r_nmask;
    int64_t *r_offsets, *r_lengths;
    int64_t r_words;
    int32_t *band;  /* per pair (SW workloads) */
    int32_t *kind;  /* per pair: 0 SW, 1 WFA (serving pool) */
    int64_t n;
} gs_batch;

/* Walk `src` from `pos`, emitting a mutated copy until `want` bases (want<0:
   until src is exhausted).  p_sub / p_indel are per-base event probabilities. */
static void mutate_walk(xs_t *r, const uint8_t *src, int64_t src_len, int64_t pos,
                        int64_t want, double p_sub, double p_indel, double geom_p,
                        buf_t *out, xs_t *fill)
{
    for (;;) {
        if (want >= 0 && out->n >= want)
            break;
        if (pos >= src_len) {
            if (want < 0)
                break;
            bput(out, ACGT[xs_next(fill) >> 62]); /* ran off the source */
            continue;
        }
        double u = xs_unif(r);
        if (u < p_sub) {
            int b = 0;
            switch (src[pos]) {
            case 'C': b = 1; break;
            case 'G': b = 2; break;
            case 'T': b = 3; break;
            default: b = 0; break;
            }
            bput(out, ACGT[(b + 1 + xs_int(r, 3)) & 3]);
            pos++;
        } else if (u < p_sub + p_indel) {
            int64_t L = xs_geom(r, geom_p);
            if (xs_next(r) >> 63) { /* insertion */
                for (int64_t k = 0; k < L; ++k)
                    bput(out, ACGT[xs_next(r) >> 62]);
            } else { /* deletion */
                pos += L;
            }
        } else {
            bput(out, src[pos]);
            pos++;
        }
    }
    if (want >= 0 && out->n > want)
        out->n = want;
}

static void add_n_runs(xs_t *r, uint8_t *s, int64_t len)
{
    for (int64_t i = 0; i < len; ++i) {
        if (xs_unif(r) < 0.001) {
            int64_t L = xs_geom(r, 0.1);
            for (int64_t k = 0; k < L && i + k < len; ++k)
                s[i + k] = 'N';
            i += L - 1;
        }
    }
}

static uint8_t *random_genome(xs_t *r, int64_t n)
{
    uint8_t *g = (uint8_t *)malloc((size_t)n);
    for (int64_t i = 0; i < n; i += 32) {
        uint64_t v = xs_next(r);
        for (int k = 0; k < 32 && i + k < n; ++k)
            g[i + k] = ACGT[(v >> (2 * k)) & 3];
    }
    return g;
}

static void finish(gs_batch *o, sb_t *q, sb_t *rb, int32_t *band, int32_t *kind, int64_t n)
{
    o->q_packed = q->packed; o->q_nmask = q->nmask;
    o->q_offsets = q->offsets; o->q_lengths = q->lengths; o->q_words = q->n_words;
    o->r_packed = rb->packed; o->r_nmask = rb->nmask;
    o->r_offsets = rb->offsets; o->r_lengths = rb->lengths; o->r_words = rb->n_words;
    o->band = band; o->kind = kind; o->n = n;
}

/* Returns 0 on success, -1 for an unknown workload id. `param` is the fixed
   length for workload 100 (ignored otherwise). */
int gs_generate(int workload, int64_t n, uint64_t seed, int64_t param, gs_batch *out)
{
    memset(out, 0, sizeof *out);
    xs_t rng, aux;
    xs_seed(&rng, seed);
    xs_seed(&aux, seed ^ 0x5DEECE66Dull);
    sb_t q, rb;
    memset(&q, 0, sizeof q);
    memset(&rb, 0, sizeof rb);
    int32_t *band = (int32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
    int32_t *kind = (int32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
    buf_t a = {0}, b = {0};

    if (workload == 0 || workload == 1) {
        int64_t glen = workload == 0 ? 1000000 : 10000000;
        uint8_t *g = random_genome(&rng, glen);
        for (int64_t i = 0; i < n; ++i) {
            int64_t origin = 25 + xs_int(&rng, glen - 25 - 175 - 1024);
            a.n = 0;
            mutate_walk(&rng, g, glen, origin, 150, 0.02, 0.005, 0.5, &a, &aux);
            sb_add(&q, a.p, a.n);
            sb_add(&rb, g + origin - 25, 200);
            band[i] = 32;
        }
        free(g);
    } else if (workload == 2 || workload == 4) {
        double lmax = workload == 2 ? 10000.0 : 20000.0;
        double dmin = workload == 2 ? 0.01 : 0.0, dmax = workload == 2 ? 0.10 : 0.15;
        for (int64_t i = 0; i < n; ++i) {
            double lu = log(100.0) + xs_unif(&rng) * (log(lmax) - log(100.0));
            int64_t L = (int64_t)llround(exp(lu));
            double d = dmin + xs_unif(&rng) * (dmax - dmin);
            a.n = 0;
            for (int64_t k = 0; k < L; ++k)
                bput(&a, ACGT[xs_next(&rng) >> 62]);
            b.n = 0;
            mutate_walk(&rng, a.p, a.n, 0, -1, 0.7 * d, 0.3 * d, 1.0 / 3.0, &b, &aux);
            sb_add(&q, a.p, a.n);
            sb_add(&rb, b.p, b.n);
            if (workload == 4) {
                kind[i] = (int32_t)(xs_next(&rng) >> 63);
                static const int32_t bands4[3] = {32, 64, 128};
                band[i] = bands4[xs_int(&rng, 3)];
            } else {
                band[i] = 0;
            }
        }
    } else if (workload == 3) {
        int64_t glen = 10000000;
        uint8_t *g = random_genome(&rng, glen);
        static const int32_t bands3[4] = {16, 32, 64, 128};
        for (int64_t i = 0; i < n; ++i) {
            int64_t ql = 100 + xs_int(&rng, 1901);
            int64_t tl = (int64_t)llround(1.25 * (double)ql);
            int64_t start = xs_int(&rng, glen - tl - 4096);
            double d = 0.01 + xs_unif(&rng) * 0.07;
            a.n = 0;
            mutate_walk(&rng, g, glen, start, ql, 0.7 * d, 0.3 * d, 1.0 / 3.0, &a, &aux);
            b.n = 0;
            for (int64_t k = 0; k < tl; ++k)
                bput(&b, g[start + k]);
            add_n_runs(&rng, a.p, a.n);
            add_n_runs(&rng, b.p, b.n);
            sb_add(&q, a.p, a.n);
            sb_add(&rb, b.p, b.n);
            band[i] = bands3[xs_int(&rng, 4)];
        }
        free(g);
    } else if (workload == 100) {
        /* harness.mojo:59-66: per-sequence LCG seeded by (i+1)*golden; the
           reference bench builds queries and refs with the same call, so pair
           i aligns a sequence to itself. */
        int64_t len = param > 0 ? param : 500;
        for (int64_t i = 0; i < n; ++i) {
            uint64_t state = (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull;
            a.n = 0;
            for (int64_t k = 0; k < len; ++k) {
                state = state * 6364136223846793005ull + 1442695040888963407ull;
                bput(&a, ACGT[(state >> 62) & 3]);
            }
            sb_add(&q, a.p, a.n);
            sb_add(&rb, a.p, a.n);
            band[i] = 32;
        }
    } else {
        free(band);
        free(kind);
        return -1;
    }
    free(a.p);
    free(b.p);
    finish(out, &q, &rb, band, kind, n);
    return 0;
}

void gs_free(gs_batch *o)
{
    free(o->q_packed); free(o->q_nmask); free(o->q_offsets); free(o->q_lengths);
    free(o->r_packed); free(o->r_nmask); free(o->r_offsets); free(o->r_lengths);
    free(o->band); free(o->kind);
    memset(o, 0, sizeof *o);
}
