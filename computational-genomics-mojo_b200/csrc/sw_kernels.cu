// sw_kernels.cu -- banded Smith-Waterman on sm_100a.
//
// Computes smith_waterman_banded (genomics/cpu/align_cpu.mojo:229-309)
// bit-exactly: score plus the first maximum cell in row-major order.
//
// Band coordinates: row qi (query position), column j in [0, 2B],
// ri = qi - B + j.  Cell (qi, j) reads diag (qi-1, j), up (qi-1, j+1) and
// left (qi, j-1) (align_cpu.mojo:277-279); E extends along the row from the
// left cell's E and opens from up (:282-283); F opens from the left H with
// no extension (:287).
//
// Register kernel (sw_band_kernel<B, G, K>): G lanes of a warp own one pair;
// lane l owns band columns [l*K, l*K + K) and keeps their H values in
// registers.  Lane l processes row t - l at step t: its first column takes
// the left neighbour's last column of the same row (computed by lane l-1 one
// step earlier, passed by warp shuffle) and its last column takes as "up"
// the right neighbour's first column of the previous row (computed by lane
// l+1 in the first phase of the same step, passed by shuffle).  With G == 1
// a thread owns the whole band row and no shuffles run.
//
// Exactness of the register kernel rests on three facts, valid when
// gap_extend <= 0, gap_open + gap_extend <= 0 and mismatch <= 0 (the host
// checks these and otherwise uses the literal kernel):
//  1. E only influences H through max(E, 0), and with gap_extend <= 0 a
//     non-positive E never becomes positive along the row, so carrying
//     E+ = max(E, 0) reproduces every H.  The reference's -1000000 start of
//     the E chain at j == 0 and the zero E of a skipped cell (:282) both
//     become E+ = 0 on the left boundary.
//  2. Cells left of the reference start (ri < 0) are skipped (zero) in the
//     reference; giving them a never-matching base makes the recurrence
//     produce exactly zero there, so no per-cell masking is needed.
//  3. Cells past the reference end (ri >= rlen) or past the query end never
//     feed a cell inside the matrix (every dependency has column <= ri and
//     row <= qi), so they are computed but excluded from the maximum.
// Padding columns past 2B in the last lane are forced to zero so column 2B
// sees the out-of-band "up" value 0 (:278).
#include "gb2_internal.cuh"

namespace gb2 {

__device__ __forceinline__ void sw_cell(int32_t hdiag, int32_t hup, int32_t hleft,
                                        int32_t eleft, int32_t sub, int32_t goe,
                                        int32_t ge, int32_t &hn, int32_t &en)
{
    // E+ = max(E_left + ge, H_up + go + ge, 0)
    en = __viaddmax_s32_relu(hup, goe, eleft + ge);
    // H = max(H_diag + sub, E+, H_left + go + ge, 0)
    hn = __viaddmax_s32_relu(hleft, goe, __viaddmax_s32(hdiag, sub, en));
}

// Writes the result of one pair from the group's packed best key.
__device__ __forceinline__ void sw_store(gb2_sw_result *out, int64_t pi, uint64_t key, int B)
{
    gb2_sw_result res;
    if (key == 0) {
        res.score = 0;
        res.query_end = 0;
        res.ref_end = 0;
    } else {
        int32_t best = (int32_t)(key >> 42);
        int32_t bq = 0x1FFFFF - (int32_t)((key >> 21) & 0x1FFFFF);
        int32_t bj = 0x1FFFFF - (int32_t)(key & 0x1FFFFF);
        res.score = best;
        res.query_end = bq;
        res.ref_end = bq - B + bj;
    }
    out[pi] = res;
}

template <int B, int G, int K>
__global__ void __launch_bounds__(128)
sw_band_kernel(SeqView q, SeqView r, SwParams p, PairList pl, gb2_sw_result *__restrict__ out)
{
    int64_t n;
    const int32_t *__restrict__ queue = pairs_resolve(pl, n);
    int *const queue_counter = pl.counter;
    constexpr int W = 2 * B + 1;
    static_assert(G * K >= W, "band does not fit");
    static_assert(G == 1 || K >= 2, "pipelined lanes need two columns");
    static_assert(32 % G == 0, "G divides the warp");
    constexpr int CPAD = W - (G - 1) * K;  // first padding column of the last lane
    static_assert(CPAD >= 1 && CPAD <= K, "G is not minimal");
    constexpr int NW = (K + 31) / 32;  // 64-bit window words per lane
    constexpr int PAIRS_PER_WARP = 32 / G;

    const int lane = threadIdx.x & 31;
    const int gl = lane % G;
    const int gw = lane / G;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (gw * G));
    const int warps_per_block = blockDim.x >> 5;
    const int64_t warp_global = (int64_t)blockIdx.x * warps_per_block + (threadIdx.x >> 5);
    const int64_t warps_total = (int64_t)gridDim.x * warps_per_block;

    const int32_t goe = p.go + p.ge;
    const int32_t ge = p.ge;
    const int32_t m = p.match, mm = p.mismatch;

    int64_t base = warp_global * PAIRS_PER_WARP;
    for (;;) {
        if (queue_counter) {
            int64_t b0 = 0;
            if (lane == 0)
                b0 = atomicAdd(queue_counter, PAIRS_PER_WARP);
            base = __shfl_sync(0xffffffffu, b0, 0);
        }
        if (base >= n)
            break;
        const int64_t slot = base + gw;
        if (slot < n) {
            const int64_t pi = queue ? (int64_t)queue[slot] : slot;
            const int64_t qoff = q.offsets[pi] - q.word_base;
            const int64_t roff = r.offsets[pi] - r.word_base;
            const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];

            int32_t H[K];
#pragma unroll
            for (int c = 0; c < K; ++c)
                H[c] = 0;
            int32_t h_in = 0, e_in = 0;
            int32_t best = 0, bq = 0, bj = 0;
            const int steps = qlen > 0 ? qlen + G - 1 : 0;
            for (int t = 0; t < steps; ++t) {
                const int qi = t - gl;
                const bool row_live = (qi >= 0) && (qi < qlen);
                const int64_t ri0 = (int64_t)qi - B + gl * K;
                uint64_t eq[NW];
                if (row_live) {
                    const uint64_t qw = __ldg(q.packed + qoff + (qi >> 5));
                    const uint64_t qb = (qw >> (62 - 2 * (qi & 31))) & 3u;
                    const uint64_t qrep = qb * 0x5555555555555555ull;
                    // NW+1 consecutive words cover the K-base window at ri0
                    const int64_t w = roff + (ri0 >> 5);
                    const int sh = (int)(ri0 & 31) * 2;
                    uint64_t words[NW + 1];
#pragma unroll
                    for (int i = 0; i <= NW; ++i) {
                        int64_t wi = w + i;
                        wi = wi < 0 ? 0 : (wi >= r.n_words ? r.n_words - 1 : wi);
                        words[i] = __ldg(r.packed + wi);
                    }
#pragma unroll
                    for (int i = 0; i < NW; ++i) {
                        const uint64_t win =
                            sh ? ((words[i] << sh) | (words[i + 1] >> (64 - sh))) : words[i];
                        const uint64_t x = win ^ qrep;
                        eq[i] = ~(x | (x >> 1)) & 0x5555555555555555ull;
                    }
                    if (ri0 < 0) {  // columns before the reference start never match
                        const int64_t nneg = -ri0;
#pragma unroll
                        for (int i = 0; i < NW; ++i) {
                            const int64_t cnt = nneg - 32 * i;
                            if (cnt >= 32)
                                eq[i] = 0;
                            else if (cnt > 0)
                                eq[i] &= (~0ull) >> (2 * cnt);
                        }
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < NW; ++i)
                        eq[i] = 0;
                }

                // phase 1: first column
                int32_t hn, en;
                {
                    const int32_t sub = ((eq[0] >> 62) & 1u) ? m : mm;
                    const int32_t hup = (K > 1) ? H[K > 1 ? 1 : 0] : 0;
                    sw_cell(H[0], hup, h_in, e_in, sub, goe, ge, hn, en);
                    if (CPAD == 0 && gl == G - 1)
                        hn = 0;
                    H[0] = hn;
                }
                int32_t up_next = 0;
                if (G > 1) {
                    up_next = __shfl_down_sync(gmask, hn, 1, G);
                    if (gl == G - 1)
                        up_next = 0;
                }
                int32_t hl = hn, el = en;
                // phase 2: remaining columns, left to right
#pragma unroll
                for (int c = 1; c < K; ++c) {
                    const int32_t sub =
                        ((eq[c >> 5] >> (62 - 2 * (c & 31))) & 1u) ? m : mm;
                    const int32_t hup = (c + 1 < K) ? H[c + 1 < K ? c + 1 : c] : up_next;
                    sw_cell(H[c], hup, hl, el, sub, goe, ge, hn, en);
                    if (c >= CPAD && gl == G - 1)
                        hn = 0;
                    H[c] = hn;
                    hl = hn;
                    el = en;
                }
                if (G > 1) {
                    h_in = __shfl_up_sync(gmask, hl, 1, G);
                    e_in = __shfl_up_sync(gmask, el, 1, G);
                    if (gl == 0) {
                        h_in = 0;
                        e_in = 0;
                    }
                }
                // first maximum of this row inside the matrix: key = H*256 + (255-c)
                if (row_live) {
                    int32_t rk = 0;
                    if (ri0 + K - 1 < rlen) {
#pragma unroll
                        for (int c = 0; c < K; ++c)
                            rk = max(rk, H[c] * 256 + (255 - c));
                    } else {
                        const int64_t lim = (int64_t)rlen - ri0;  // columns c < lim are inside
#pragma unroll
                        for (int c = 0; c < K; ++c)
                            rk = max(rk, (c < lim) ? H[c] * 256 + (255 - c) : 0);
                    }
                    if ((rk >> 8) > best) {
                        best = rk >> 8;
                        bq = qi;
                        bj = gl * K + 255 - (rk & 255);
                    }
                }
            }
            uint64_t key = 0;
            if (best > 0)
                key = ((uint64_t)best << 42) | ((uint64_t)(0x1FFFFF - bq) << 21) |
                      (uint64_t)(0x1FFFFF - bj);
#pragma unroll
            for (int off = 1; off < G; off <<= 1) {
                const uint64_t o = __shfl_xor_sync(gmask, key, off, G);
                key = o > key ? o : key;
            }
            if (gl == 0)
                sw_store(out, pi, key, B);
        }
        if (!queue_counter)
            base += warps_total * PAIRS_PER_WARP;
    }
}

// ---------------------------------------------------------------------------
// Packed int16x2 kernel (sw_pack16_kernel<B>): one thread per pair, two cells
// per 32-bit register, one DPX instruction advancing both.
//
// Band columns 0..B live in the low halves, columns B+1..2B in the high
// halves of R = B+1 registers; the high half of the last register is a
// padding column held at H = 0 (it is the out-of-band "up" of column 2B).
// At step t the low halves hold row t and the high halves row t-1, so the
// two cells of a register are never each other's neighbours:
//   low  (t, h):      diag/up from the same half of registers h, h+1 of step
//                     t-1; up of h = B is the high half of register 0 (row
//                     t-1, column B+1), computed earlier in this step;
//   high (t-1, B+1+h): diag/up from the same half of step t-1; left of h = 0
//                     is the low half of register B of step t-1 (row t-1,
//                     column B).
// Values: registers hold H; the E chain is carried as E - (go+ge), so
//   E' = max(E'_left + ge, H_up),
//   H  = max(H_diag + sub - (go+ge), E', H_left, -(go+ge)) + (go+ge).
// Without the max(E, 0) clamp E differs from the reference's E only in
// non-positive values, which never reach H (H takes max(.., 0)); the
// -1000000 start of the chain at column 0 becomes a large negative value.
// Bits: H <= 511 in every cell (the host checks match*min(qlen, rlen)), all
// terms stay inside int16, the first-maximum key H*128 + (127-column) fits
// an unsigned 16-bit half, and the per-half subtract of |go+ge| cannot
// borrow because H' >= |go+ge|.
//
// Pipe balance.  The three DPX max instructions per register run on the
// integer ALU pipe, which this recurrence saturates; the FMA pipe (integer
// multiply-add) is a separate pipe of the same width.  So every step that a
// multiply-add can do runs there, with multipliers passed as kernel
// arguments (Pack16Consts) so the compiler cannot turn them back into
// shifts:
//  - the substitution score of both cells of a register is one mad.hi: the
//    equality bits of the two cells sit at bits p and p+16 of a word, and
//    hi32(bits * ((match-mismatch) << (32-p))) + (mismatch-(go+ge)) in both
//    halves is exact while (match-mismatch) << (32-p) fits 32 bits (p >= 8
//    here; the host requires match-mismatch <= 255);
//  - the -(go+ge) subtract, the key H*128 + tag, the two-bit shifts that
//    slide the reference window and the previous row's equality bits, and
//    the one-bit shift of the equality test are multiply-adds or mad.hi.
// Sequences are read as 16-base (32-bit) words, reloaded every 16 rows; the
// reference word entering the window and the query word are consumed two
// bits per row by multiplication.
// ---------------------------------------------------------------------------
// Constants of sw_pack16_kernel, built by the host from SwParams.  The
// multipliers (1, 4, 128, 256, 2^31 and the shifted score difference) are
// kernel arguments rather than literals so that the multiply-adds using them
// stay multiply-adds.
struct Pack16Consts {
    uint32_t one, x4, x128, x256, half;
    uint32_t dm[4];  // (match - mismatch) << 18, 20, 22, 24
    uint32_t mmg2;   // mismatch - (go+ge) in both halves
    uint32_t neg_g2; // minus -(go+ge) in both halves, mod 2^32
    uint32_t ge2;    // ge in both halves
    uint32_t ng2;    // -(go+ge) in both halves
    // the wide-key multipliers stay last: with them placed before x128 the narrow
    // band-32 kernel measured 9% slower (665 vs 610 us per 262,144-pair launch,
    // same registers)
    uint32_t x8, x32;
};

__device__ __forceinline__ uint32_t mad_hi_u32(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// (a << 2) | (b >> 30) as two multiply-adds (x4 == 4).
__device__ __forceinline__ uint32_t shl2_in(uint32_t a, uint32_t b, uint32_t x4)
{
    return a * x4 + mad_hi_u32(b, x4, 0u);
}

// 16-base word k (bases 16k..16k+15, first base in the top two bits) of the
// 2-bit MSB-first sequence starting at 64-bit word `off`; k is clamped into
// the packed array (the clamped words are never read by an in-matrix cell).
__device__ __forceinline__ uint32_t seq_word16(const SeqView &s, int64_t off, int64_t k)
{
    int64_t i = 2 * off + (k ^ 1);
    const int64_t last = 2 * s.n_words - 1;
    i = i < 0 ? 0 : (i > last ? last : i);
    return __ldg(reinterpret_cast<const uint32_t *>(s.packed) + i);
}

// One step of sw_pack16_kernel over all R registers.  eq[k] / bw[k]: the
// equality bits (bit 30-2c for column 16k+c) of row t and of row t-1 shifted
// so column B+1+h sits where column h does.  MASK = false when every cell of
// the step lies inside the matrix (the common case); MASK = true zeroes the
// first-maximum keys of cells past the query or reference end.  Returns the
// packed row keys: low half row t, high half row t-1.
//
// WIDE keys (scores up to 4094, bands 16..128): the key H*128 + column of the
// narrow form needs H <= 511 and 2B+1 <= 128 columns.  The wide form keys a
// cell as H*8 + (7 - h%8) (no carry between halves while H <= 8191), takes
// the maximum over each group of 8 registers, and turns each group's maximum
// into relu(gk - 8*base) with one DPX instruction, base = the best score of
// the rows already resolved: a cell can only become the new best when
// H > base, and then H - base <= 2*match (a row's maximum exceeds the
// previous row's by at most `match`).  The group key
//   (H - base) * 256 + (31 - group) * 8 + (7 - h%8)
// fits 16 bits for match <= 127, and its maximum over the groups is the
// first maximum of the half; group keys below 256 mean "nothing above base".
// Per register this costs what the narrow key costs (one multiply-add and
// half a 3-way max); the DPX relu, two logic ops and a multiply-add run once
// per group.
template <int B, bool MASK, bool WIDE>
__device__ __forceinline__ uint32_t pack16_cells(uint32_t (&Hr)[B + 1], const uint32_t *eq,
                                                 const uint32_t *bw, uint32_t &e_last, int limL,
                                                 int limH, const Pack16Consts &c,
                                                 uint32_t negbase8)
{
    constexpr int NL = B + 1, R = NL;
    // Bands 64 and 128 are register-bound to 12 and 8 warps per SM, too few to
    // hide the latency of the left-to-right chain through a row: there the
    // H update is grouped so that only the 3-way max waits on the left
    // neighbour (two dependent instructions per register instead of three).
    // Measured on 1,000,000 reads: band 128 2,723 -> 2,901 GCUPS, band 64
    // 3,613 -> 3,655; the narrow bands 16 and 32 (20 warps per SM) are 4%
    // faster with the other grouping.
    constexpr bool SHORT_CHAIN = B >= 64;
    const uint32_t SENT = 0x0000C000u;
    uint32_t hl = Hr[R - 1] << 16;                    // low: band edge 0; high: H(t-1, B)
    uint32_t el = __byte_perm(SENT, e_last, 0x5410);  // low: chain start; high: E'(t-1, B)
    uint32_t h0new = 0;
    uint32_t rk = 0, kpend = 0;
    uint32_t gacc = 0, gpend = 0, g2pend = 0;  // WIDE: group maximum, pending keys
#pragma unroll
    for (int h = 0; h < R; ++h) {
        const int k = h >> 4, j = h & 15, jj = h & 7;
        // cells 8*(h>>3) .. +7 of both halves at bits 14-2*jj and 30-2*jj
        const uint32_t wsel = (j < 8) ? __byte_perm(eq[k], bw[k], 0x7632)
                                      : __byte_perm(eq[k], bw[k], 0x5410);
        const uint32_t wv = (jj < 4) ? wsel : wsel * c.x256;  // cells 4..7 up to bits 14..8
        const int pos = 14 - 2 * (jj & 3);
        const uint32_t sub =
            mad_hi_u32(wv & ((1u << pos) | (1u << (pos + 16))), c.dm[jj & 3], c.mmg2);
        const uint32_t up = (h + 1 < R) ? Hr[h + 1 < R ? h + 1 : h] : (h0new >> 16);
        const uint32_t e = __viaddmax_s16x2(el, c.ge2, up);
        uint32_t hn;
        if (!SHORT_CHAIN) {
            const uint32_t tt = __vimax3_s16x2(e, hl, c.ng2);
            hn = __viaddmax_s16x2(Hr[h], sub, tt) * c.one + c.neg_g2;
        } else {
            const uint32_t a = __viaddmax_s16x2(Hr[h], sub, e);
            hn = __vimax3_s16x2(a, hl, c.ng2) * c.one + c.neg_g2;
        }
        hl = hn;
        if (h == R - 1)
            hn &= 0x0000FFFFu;  // padding column stays 0
        if (h == 0)
            h0new = hn;
        Hr[h] = hn;
        el = e;
        if (!WIDE) {
            uint32_t key =
                hn * c.x128 + (((uint32_t)(127 - h)) | ((uint32_t)(127 - NL - h) << 16));
            if (MASK)
                key &= (h < limL ? 0x0000FFFFu : 0u) | (h < limH ? 0xFFFF0000u : 0u);
            if (h & 1)
                rk = __vimax3_u16x2(rk, kpend, key);
            else
                kpend = key;
        } else {
            const int i = h & 7, g = h >> 3;
            const uint32_t t8 = 7u - (uint32_t)i;
            uint32_t key = hn * c.x8 + (t8 | (t8 << 16));
            if (MASK)
                key &= (h < limL ? 0x0000FFFFu : 0u) | (h < limH ? 0xFFFF0000u : 0u);
            if (i == 0)
                gacc = key;
            else if (i & 1)
                gpend = key;
            else
                gacc = __vimax3_u16x2(gacc, gpend, key);
            if (i == 7 || h == R - 1) {
                if (i & 1)
                    gacc = __vimax3_u16x2(gacc, gpend, gpend);
                const uint32_t ck = __viaddmax_s16x2_relu(gacc, negbase8, 0u);
                const uint32_t cg = (uint32_t)((31 - g) * 8) * 0x00010001u;
                const uint32_t k2 = (ck & 0xFFF8FFF8u) * c.x32 + ((ck & 0x00070007u) | cg);
                if (g & 1)
                    rk = __vimax3_u16x2(rk, g2pend, k2);
                else
                    g2pend = k2;
            }
        }
    }
    if (!WIDE) {
        if ((R - 1) % 2 == 0)
            rk = __vimax3_u16x2(rk, kpend, kpend);
    } else {
        constexpr int NG = (R + 7) / 8;
        if ((NG - 1) % 2 == 0)
            rk = __vimax3_u16x2(rk, g2pend, g2pend);
    }
    e_last = el;
    return rk;
}

// Band 128 is register-bound to two blocks per SM either way; with the
// minimum-blocks hint of 1 the compiler schedules it in 254 registers instead
// of 251 and the kernel measured 6% faster (2,734 vs 2,583 GCUPS).  The other
// widths keep the default schedule (hint 0).
template <int B, bool WIDE>
__global__ void __launch_bounds__(128, (B == 128) ? 1 : 0)
sw_pack16_kernel(SeqView q, SeqView r, Pack16Consts c, PairList pl, gb2_sw_result *__restrict__ out)
{
    static_assert(B % 16 == 0, "band must be a multiple of 16");
    constexpr int W = 2 * B + 1;
    constexpr int NL = B + 1;           // columns in low halves
    constexpr int R = NL;               // registers
    constexpr int NE = (W + 15) / 16;   // 16-column equality words of one row
    constexpr int BW0 = NL / 16;        // first word of columns B+1.. (offset one column)
    constexpr int NBW = B / 16;         // shifted words of the previous row
    constexpr int RW0 = NE - B / 16;    // 16-base word entering the window at t = 0
    static_assert(WIDE || W <= 127, "column index must fit the narrow key");
    static_assert(!WIDE || (R + 7) / 8 <= 32, "group index must fit the wide key");
    static_assert(NL % 16 == 1 && BW0 + NBW < NE, "word layout");

    int64_t n;
    const int32_t *__restrict__ queue = pairs_resolve(pl, n);
    int *const queue_counter = pl.counter;
    const int lane = threadIdx.x & 31;
    const int warps_per_block = blockDim.x >> 5;
    const int64_t warp_global = (int64_t)blockIdx.x * warps_per_block + (threadIdx.x >> 5);
    const int64_t warps_total = (int64_t)gridDim.x * warps_per_block;
    const uint32_t SENT = 0x0000C000u;  // -16384 in the low half

    int64_t base = warp_global * 32;
    for (;;) {
        if (queue_counter) {
            int64_t b0 = 0;
            if (lane == 0)
                b0 = atomicAdd(queue_counter, 32);
            base = __shfl_sync(0xffffffffu, b0, 0);
        }
        if (base >= n)
            break;
        const int64_t slot = base + lane;
        if (slot < n) {
            const int64_t pi = queue ? (int64_t)queue[slot] : slot;
            const int64_t qoff = q.offsets[pi] - q.word_base;
            const int64_t roff = r.offsets[pi] - r.word_base;
            const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
            uint32_t Hr[R];
#pragma unroll
            for (int h = 0; h < R; ++h)
                Hr[h] = 0;
            uint32_t ep[NE];  // equality bits of the previous row
#pragma unroll
            for (int i = 0; i < NE; ++i)
                ep[i] = 0;
            // The reference window of row t, r[t-B .. t-B+16*NE), one 16-base word
            // per entry, slid by one base per row; the base entering at the bottom
            // is the top of `rw`, the word of positions t-B+16*NE.., reloaded every
            // 16 rows (t-B+16*NE is a multiple of 16 exactly when t is).  Words
            // before the reference start are zero and masked below.
            uint32_t win[NE];
#pragma unroll
            for (int i = 0; i < NE; ++i)
                win[i] = (i < B / 16) ? 0u : seq_word16(r, roff, i - B / 16);
            uint32_t e_last = SENT;
            uint32_t saved_lowkey = 0, bestkey = 0, thr = 127;
            int32_t bq = 0;
            // WIDE: best score, its column, and the base the saved key was taken at
            int32_t best = 0, bcol = 0, base_prev = 0;
            uint32_t qw = 0, rw = 0;
            uint32_t qn = seq_word16(q, qoff, 0), rn = seq_word16(r, roff, RW0);  // next words
            const int steps = qlen > 0 ? qlen + 1 : 0;
            const int full_end = min(qlen, rlen - B + 1);  // rows t < full_end lie inside
            for (int t = 0; t < steps; ++t) {
                if ((t & 15) == 0) {  // words of rows t..t+15; fetch the following ones
                    qw = qn;
                    rw = rn;
                    qn = seq_word16(q, qoff, (t >> 4) + 1);
                    rn = seq_word16(r, roff, (t >> 4) + RW0 + 1);
                }
                // equality bits of row t against its window r[t-B .. t+B]
                const uint32_t qrep = mad_hi_u32(qw, c.x4, 0u) * 0x55555555u;
                qw *= c.x4;
                uint32_t eq[NE];
#pragma unroll
                for (int i = 0; i < NE; ++i) {
                    const uint32_t x = win[i] ^ qrep;
                    eq[i] = ~(x | mad_hi_u32(x, c.half, 0u)) & 0x55555555u;
                }
                if (t < B) {  // columns before the reference start never match
#pragma unroll
                    for (int i = 0; i < NE; ++i) {
                        const int cnt = B - t - 16 * i;
                        if (cnt >= 16)
                            eq[i] = 0;
                        else if (cnt > 0)
                            eq[i] &= 0xFFFFFFFFu >> (2 * cnt);
                    }
                }
                // slide the window one base for row t+1
#pragma unroll
                for (int i = 0; i + 1 < NE; ++i)
                    win[i] = shl2_in(win[i], win[i + 1], c.x4);
                win[NE - 1] = shl2_in(win[NE - 1], rw, c.x4);
                rw *= c.x4;
                // previous row's bits, shifted so column NL+h sits where column h does;
                // the last word holds only the padding column
                uint32_t bw[NBW + 1];
#pragma unroll
                for (int i = 0; i < NBW; ++i)
                    bw[i] = shl2_in(ep[BW0 + i], ep[BW0 + i + 1], c.x4);
                bw[NBW] = 0;
                const bool full = t >= 1 && t < full_end;
                int limL = 0, limH = 0;
                if (!full) {
                    if (t < qlen)
                        limL = max(0, min(NL, rlen - (t - B)));
                    if (t >= 1 && t - 1 < qlen)
                        limH = max(0, min(R, rlen - (t - 1 - B + NL)));
                }
                // WIDE keys are relative to the best score of rows <= t-2
                const uint32_t negbase8 = (uint32_t)(uint16_t)(-8 * best) * 0x00010001u;
                const uint32_t rk =
                    full ? pack16_cells<B, false, WIDE>(Hr, eq, bw, e_last, 0, 0, c, negbase8)
                         : pack16_cells<B, true, WIDE>(Hr, eq, bw, e_last, limL, limH, c,
                                                       negbase8);
                if (!WIDE) {
                    // row t-1 is complete: its first half came one step earlier; a key
                    // above thr = bestkey | 127 has a larger H than the best so far
                    const uint32_t rowkey = max(saved_lowkey, rk >> 16);
                    if (rowkey > thr) {
                        thr = rowkey | 127u;
                        bestkey = rowkey;
                        bq = t - 1;
                    }
                    saved_lowkey = rk & 0xFFFFu;
                } else {
                    // the saved low half of row t-1 was keyed against base_prev: rebase
                    // it to this step's base; then the low half wins ties (its columns
                    // come first)
                    const uint32_t dsh = (uint32_t)(best - base_prev) << 8;
                    const uint32_t sl = saved_lowkey >= dsh + 256u ? saved_lowkey - dsh : 0u;
                    const uint32_t hi = rk >> 16;
                    const int32_t dl = (int32_t)(sl >> 8), dh = (int32_t)(hi >> 8);
                    base_prev = best;
                    if (dl > 0 || dh > 0) {
                        if (dl >= dh) {
                            best += dl;
                            bcol = 255 - (int32_t)(sl & 255u);
                        } else {
                            best += dh;
                            bcol = NL + 255 - (int32_t)(hi & 255u);
                        }
                        bq = t - 1;
                    }
                    saved_lowkey = rk & 0xFFFFu;
                }
#pragma unroll
                for (int i = 0; i < NE; ++i)
                    ep[i] = eq[i];
            }
            if (!WIDE) {
                best = (int32_t)(bestkey >> 7);
                bcol = 127 - (int32_t)(bestkey & 127u);
            }
            gb2_sw_result res;
            res.score = best;
            res.query_end = best > 0 ? bq : 0;
            res.ref_end = best > 0 ? bq - B + bcol : 0;
            out[pi] = res;
        }
        if (!queue_counter)
            base += warps_total * 32;
    }
}

// Literal per-pair kernel: one thread per pair, int64 arithmetic, rows in
// global scratch.  Statement order follows align_cpu.mojo:239-309 exactly,
// so it is exact for every configuration and band.
__global__ void __launch_bounds__(128)
sw_literal_kernel(SeqView q, SeqView r, SwParams p, int32_t band, const int32_t *__restrict__ bands,
                  PairList pl, gb2_sw_result *__restrict__ out, int64_t *__restrict__ scratch,
                  int64_t stride)
{
    int64_t n;
    const int32_t *__restrict__ queue = pairs_resolve(pl, n);
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    int64_t *hp = scratch + tid * stride;
    for (int64_t slot = tid; slot < n; slot += nth) {
        const int64_t pi = queue ? (int64_t)queue[slot] : slot;
        const int64_t b = bands ? bands[pi] : band;
        const int64_t width = 2 * b + 1;
        int64_t *hc = hp + width, *ec = hp + 2 * width;
        const int64_t qlen = q.lengths[pi], rlen = r.lengths[pi];
        const uint64_t *qw = q.packed + (q.offsets[pi] - q.word_base);
        const uint64_t *rw = r.packed + (r.offsets[pi] - r.word_base);
        int64_t best = 0, bq = 0, br = 0;
        if (width > 0) {
            for (int64_t j = 0; j < width; ++j)
                hp[j] = 0;
            for (int64_t qi = 0; qi < qlen; ++qi) {
                for (int64_t j = 0; j < width; ++j) {
                    hc[j] = 0;
                    ec[j] = 0;
                }
                const int64_t qb = (int64_t)((qw[qi >> 5] >> (62 - 2 * (qi & 31))) & 3u);
                for (int64_t off = 0; off < width; ++off) {
                    const int64_t ri = qi - b + off;
                    if (ri < 0 || ri >= rlen)
                        continue;
                    const int64_t rb = (int64_t)((rw[ri >> 5] >> (62 - 2 * (ri & 31))) & 3u);
                    const int64_t sub = (qb == rb) ? p.match : p.mismatch;
                    const int64_t h_diag = hp[off];
                    const int64_t h_up = (off + 1 < width) ? hp[off + 1] : 0;
                    const int64_t h_left = (off > 0) ? hc[off - 1] : 0;
                    int64_t e1 = (off > 0) ? ec[off - 1] + p.ge : -1000000LL;
                    int64_t e2 = h_up + p.go + p.ge;
                    const int64_t e_val = e1 > e2 ? e1 : e2;
                    const int64_t f_val = h_left + p.go + p.ge;
                    int64_t cell = h_diag + sub;
                    cell = cell > e_val ? cell : e_val;
                    cell = cell > f_val ? cell : f_val;
                    cell = cell > 0 ? cell : 0;
                    hc[off] = cell;
                    ec[off] = e_val;
                    if (cell > best) {
                        best = cell;
                        bq = qi;
                        br = ri;
                    }
                }
                for (int64_t j = 0; j < width; ++j)
                    hp[j] = hc[j];
            }
        }
        gb2_sw_result res;
        res.score = (int32_t)best;
        res.query_end = (int32_t)bq;
        res.ref_end = (int32_t)br;
        out[pi] = res;
    }
}

// Naive baseline (GB2_FLAG_NAIVE): one 128-thread block per pair, launched
// over all pairs in input order with no planning, as the reference's
// launch_banded_sw does (genomics/gpu/align_gpu.mojo:482-492) -- but computing
// the CPU recurrence exactly.  Cell (qi, j) of the band runs at step
// s = 2*qi + j: its diag (qi-1, j) ran at s-2, its up (qi-1, j+1) and left
// (qi, j-1) at s-1, so the cells of one step (one parity of j) are
// independent and one row of H and E per band column, in shared memory, holds
// every value a step reads; a barrier separates the steps.  Skipped cells
// (reference position outside [0, rlen)) hold 0 as the reference's reset rows
// do (align_cpu.mojo:261-268).  int32 values (the host bounds every score).
__global__ void __launch_bounds__(128)
sw_naive_kernel(SeqView q, SeqView r, SwParams p, int32_t band, const int32_t *__restrict__ bands,
                int64_t n, gb2_sw_result *__restrict__ out)
{
    extern __shared__ int32_t nsm[];
    __shared__ unsigned long long red[4];
    const int64_t pi = blockIdx.x;
    if (pi >= n)
        return;
    const int32_t b = bands ? bands[pi] : band;
    const int32_t W = 2 * b + 1;
    int32_t *const Hs = nsm;
    int32_t *const Es = nsm + W;
    const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
    const uint64_t *qw = q.packed + (q.offsets[pi] - q.word_base);
    const uint64_t *rw = r.packed + (r.offsets[pi] - r.word_base);
    for (int32_t j = threadIdx.x; j < W; j += blockDim.x) {
        Hs[j] = 0;
        Es[j] = 0;
    }
    __syncthreads();
    unsigned long long best = 0;  // H << 42 | (2^21-1 - qi) << 21 | (2^21-1 - j)
    const int32_t steps = qlen > 0 ? 2 * (qlen - 1) + W : 0;
    const int32_t goe = p.go + p.ge;
    for (int32_t st = 0; st < steps; ++st) {
        // active columns: parity of st, qi = (st - j) / 2 in [0, qlen)
        const int32_t jlo = max(st & 1, st - 2 * (qlen - 1));
        const int32_t jhi = min(W - 1, st);
        for (int32_t j = jlo + 2 * (int32_t)threadIdx.x; j <= jhi; j += 2 * (int32_t)blockDim.x) {
            const int32_t qi = (st - j) >> 1;
            const int32_t ri = qi - b + j;
            int32_t h = 0, e = 0;
            if (ri >= 0 && ri < rlen) {
                const int32_t qb = (int32_t)((qw[qi >> 5] >> (62 - 2 * (qi & 31))) & 3u);
                const int32_t rb = (int32_t)((rw[ri >> 5] >> (62 - 2 * (ri & 31))) & 3u);
                const int32_t sub = qb == rb ? p.match : p.mismatch;
                const int32_t h_diag = Hs[j];
                const int32_t h_up = j + 1 < W ? Hs[j + 1] : 0;
                const int32_t h_left = j > 0 ? Hs[j - 1] : 0;
                const int32_t e1 = j > 0 ? Es[j - 1] + p.ge : -1000000;
                e = max(e1, h_up + goe);
                h = max(max(h_diag + sub, e), max(h_left + goe, 0));
                if (h > 0) {
                    const unsigned long long key =
                        ((unsigned long long)h << 42) |
                        ((unsigned long long)(0x1FFFFF - qi) << 21) |
                        (unsigned long long)(0x1FFFFF - j);
                    best = key > best ? key : best;
                }
            }
            Hs[j] = h;
            Es[j] = e;
        }
        __syncthreads();
    }
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
    }
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i)
            best = red[i] > best ? red[i] : best;
        sw_store(out, pi, best, b);
    }
}

cudaError_t launch_sw_naive(SeqView q, SeqView r, SwParams p, int32_t band, const int32_t *bands,
                            int32_t max_band, int64_t n, gb2_sw_result *out, cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    if (n > 0x7fffffff || max_band > kSwNaiveMaxBand)
        return cudaErrorInvalidValue;
    static const cudaError_t attr = cudaFuncSetAttribute(
        sw_naive_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)(2 * (2 * kSwNaiveMaxBand + 1) * sizeof(int32_t)));
    (void)attr;
    const size_t smem = (size_t)2 * (2 * (size_t)max_band + 1) * sizeof(int32_t);
    sw_naive_kernel<<<(unsigned)n, 128, smem, st>>>(q, r, p, band, bands, n, out);
    return cudaGetLastError();
}

template <int B, int G, int K>
static cudaError_t launch_band(SeqView q, SeqView r, SwParams p, PairList pl, gb2_sw_result *out,
                               int grid, cudaStream_t st)
{
    const int block = 128;
    const int64_t pairs_per_block = (block / 32) * (32 / G);
    int g = grid;
    if (g <= 0) {  // one pass over a host-known count
        if (pl.seg || pl.n <= 0)
            return pl.n <= 0 && !pl.seg ? cudaSuccess : cudaErrorInvalidValue;
        const int64_t need = (pl.n + pairs_per_block - 1) / pairs_per_block;
        g = (int)(need < 0x7fffffff ? need : 0x7fffffff);
    }
    sw_band_kernel<B, G, K><<<g, block, 0, st>>>(q, r, p, pl, out);
    return cudaGetLastError();
}

template <int B, int G, int K>
static int occ_band()
{
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sw_band_kernel<B, G, K>, 128, 0);
    return nb > 0 ? nb : 1;
}

template <int B, bool WIDE>
static int occ_pack16()
{
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sw_pack16_kernel<B, WIDE>, 128, 0);
    return nb > 0 ? nb : 1;
}

int sw_blocks_per_sm(int band_class, int variant)
{
    switch (band_class) {
    case 16 | kPack16: return occ_pack16<16, false>();
    case 32 | kPack16: return occ_pack16<32, false>();
    case 16 | kPackWide: return occ_pack16<16, true>();
    case 32 | kPackWide: return occ_pack16<32, true>();
    case 64 | kPackWide: return occ_pack16<64, true>();
    case 128 | kPackWide: return occ_pack16<128, true>();
    case 16: return variant == 1 ? occ_band<16, 2, 17>() : occ_band<16, 1, 33>();
    case 32:
        return variant == 1 ? occ_band<32, 2, 33>()
                            : (variant == 2 ? occ_band<32, 4, 17>() : occ_band<32, 1, 65>());
    case 64: return variant == 1 ? occ_band<64, 4, 33>() : occ_band<64, 2, 65>();
    case 128: return variant == 1 ? occ_band<128, 8, 33>() : occ_band<128, 4, 65>();
    default: return 4;
    }
}

int sw_pairs_per_block(int band_class, int variant)
{
    int G = 1;
    switch (band_class) {
    case 16 | kPack16:
    case 32 | kPack16:
    case 16 | kPackWide:
    case 32 | kPackWide:
    case 64 | kPackWide:
    case 128 | kPackWide: return 128;
    case 16: G = variant == 1 ? 2 : 1; break;
    case 32: G = variant == 1 ? 2 : (variant == 2 ? 4 : 1); break;
    case 64: G = variant == 1 ? 4 : 2; break;
    case 128: G = variant == 1 ? 8 : 4; break;
    default: return 128;
    }
    return 4 * (32 / G);
}

// variant selects (G, K) for a band class: 0 = default.
cudaError_t launch_sw(int band_class, int variant, SeqView q, SeqView r, SwParams p, int32_t band,
                      const int32_t *bands, PairList pl, gb2_sw_result *out, int64_t *scratch,
                      int64_t scratch_stride, int grid, cudaStream_t st)
{
    switch (band_class) {
    case 16 | kPack16:
    case 32 | kPack16:
    case 16 | kPackWide:
    case 32 | kPackWide:
    case 64 | kPackWide:
    case 128 | kPackWide: {
        int g = grid;
        if (g <= 0) {
            if (pl.seg || pl.n <= 0)
                return pl.n <= 0 && !pl.seg ? cudaSuccess : cudaErrorInvalidValue;
            g = (int)((pl.n + 127) / 128);
        }
        const uint32_t gg = (uint32_t)(-(p.go + p.ge)), dm = (uint32_t)(p.match - p.mismatch);
        Pack16Consts c;
        c.one = 1;
        c.x4 = 4;
        c.x8 = 8;
        c.x32 = 32;
        c.x128 = 128;
        c.x256 = 256;
        c.half = 0x80000000u;
        for (int i = 0; i < 4; ++i)
            c.dm[i] = dm << (18 + 2 * i);
        c.mmg2 = ((uint32_t)p.mismatch + gg) * 0x00010001u;
        c.neg_g2 = 0u - gg * 0x00010001u;
        c.ge2 = (uint32_t)(uint16_t)p.ge * 0x00010001u;
        c.ng2 = (uint32_t)(uint16_t)gg * 0x00010001u;
        switch (band_class) {
        case 16 | kPack16: sw_pack16_kernel<16, false><<<g, 128, 0, st>>>(q, r, c, pl, out); break;
        case 32 | kPack16: sw_pack16_kernel<32, false><<<g, 128, 0, st>>>(q, r, c, pl, out); break;
        case 16 | kPackWide: sw_pack16_kernel<16, true><<<g, 128, 0, st>>>(q, r, c, pl, out); break;
        case 32 | kPackWide: sw_pack16_kernel<32, true><<<g, 128, 0, st>>>(q, r, c, pl, out); break;
        case 64 | kPackWide: sw_pack16_kernel<64, true><<<g, 128, 0, st>>>(q, r, c, pl, out); break;
        default: sw_pack16_kernel<128, true><<<g, 128, 0, st>>>(q, r, c, pl, out); break;
        }
        return cudaGetLastError();
    }
    case 16:
        if (variant == 1)
            return launch_band<16, 2, 17>(q, r, p, pl, out, grid, st);
        return launch_band<16, 1, 33>(q, r, p, pl, out, grid, st);
    case 32:
        if (variant == 1)
            return launch_band<32, 2, 33>(q, r, p, pl, out, grid, st);
        if (variant == 2)
            return launch_band<32, 4, 17>(q, r, p, pl, out, grid, st);
        return launch_band<32, 1, 65>(q, r, p, pl, out, grid, st);
    case 64:
        if (variant == 1)
            return launch_band<64, 4, 33>(q, r, p, pl, out, grid, st);
        return launch_band<64, 2, 65>(q, r, p, pl, out, grid, st);
    case 128:
        if (variant == 1)
            return launch_band<128, 8, 33>(q, r, p, pl, out, grid, st);
        return launch_band<128, 4, 65>(q, r, p, pl, out, grid, st);
    default: {
        if (grid <= 0)
            return cudaErrorInvalidValue;  // the literal kernel needs a sized scratch grid
        sw_literal_kernel<<<grid, 128, 0, st>>>(q, r, p, band, bands, pl, out, scratch,
                                                scratch_stride);
        return cudaGetLastError();
    }
    }
}

}  // namespace gb2
