// wfa_kernels.cu -- gap-affine WFA cost on sm_100a.
//
// Computes wfa_affine_cpu (genomics/cpu/align_cpu.mojo:75-226) exactly:
//   I[s,k] = max(M[s-o-e,k-1]+1, I[s-e,k-1]+1)
//   D[s,k] = max(M[s-o-e,k+1],   D[s-e,k+1])
//   M[s,k] = max(M[s-x,k]+1, I[s,k], D[s,k]),  then extend M through matches;
// k = row - col, terminate at the first s with M[s, qlen-rlen] >= qlen, -1
// past max_error.  Offsets are never clamped (as in the reference).
//
// Equivalences used (all keep every value the reference computes):
//  * Only scores that are multiples of g = gcd(x, o, e) can hold a non-NEG
//    value, so the loop visits s = g, 2g, ... and the rings are indexed in
//    units of g.
//  * A diagonal is only visited if one of its sources is non-empty: the
//    visited interval at score s is the union of the source intervals
//    (M[s-x]; M[s-o-e] +-1; I[s-e] + 1; D[s-e] - 1) intersected with the
//    reference's [lo, hi] (widened to the target and clamped to +-max_error,
//    :158-164).  Everything outside it is NEG in the reference.
//  * NEG is a large negative number and sources are combined with plain max;
//    every value below zero is stored as NEG and every non-NEG value is
//    >= 0, so "negative" reproduces the reference's "== NEG_INF" tests
//    (:174-204) and its "row < 0" skip (:211).
//
// Ring slots live in a scratch region per warp, one int32 per diagonal
// (index k + rlen + 2).  Invariant: inside the interval [GL, GH] that a pair
// has touched, every slot position outside that slot's own interval holds
// NEG; so source reads at k-1, k, k+1 need no bounds tests.
#include <type_traits>

#include "gb2_internal.cuh"
#include "wfa_trace.cuh"

namespace gb2 {

#define WFA_NEG (-(1 << 30))

__device__ __forceinline__ int gcd_i(int a, int b)
{
    while (b) {
        int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// A sequence as 32-bit halves of its packed words (16 bases each, MSB
// first): logical half j sits at w[j ^ swz] -- swz = 0 for the shared-memory
// copy (stored high half first), 1 for the packed words in global memory
// (little-endian, so a word's high half comes second).  Logical half `last`
// is the one after the sequence's last half (a zero pad in shared memory, or
// the array's next half in global memory, clamped to the array's end).
struct SeqHalves {
    const uint32_t *w;
    int32_t last;
    uint32_t swz;
};

// 16 bases at position pos: one funnel shift of two halves (the shift
// amount is taken mod 32, so pos << 1 is (pos mod 16) * 2).  Bases past the
// sequence end never matter: matches are clamped by the remaining lengths.
// SMEM: the halves are the shared-memory copy, whose zero pad word makes the
// second half always present -- no clamp, shared addressing.
template <bool SMEM>
__device__ __forceinline__ uint32_t window16(const SeqHalves &s, int32_t pos)
{
    const int32_t j = pos >> 4;
    uint32_t hi, lo;
    if (SMEM) {
        hi = s.w[j];
        lo = s.w[j + 1];
    } else {
        hi = s.w[(uint32_t)j ^ s.swz];
        lo = s.w[(uint32_t)min(j + 1, s.last) ^ s.swz];
    }
    return __funnelshift_l(lo, hi, (uint32_t)pos << 1);
}

// Extend along diagonal k from row (align_cpu.mojo:208-219): XOR of the two
// 16-base windows, count leading zeros (32 for a full match, so the match
// length is clz / 2 either way), clamp by the remaining lengths.
template <bool SMEM>
__device__ __forceinline__ int32_t extend_run(const SeqHalves &qs, int32_t qlen,
                                              const SeqHalves &rs, int32_t rlen, int32_t row,
                                              int32_t k)
{
    if (row < 0 || row - k < 0)
        return row;
    int32_t col = row - k;
    while (row < qlen && col < rlen) {
        const uint32_t x = window16<SMEM>(qs, row) ^ window16<SMEM>(rs, col);
        const int ml = __clz((int)x) >> 1;
        const int lim = min(qlen - row, rlen - col);
        if (ml >= lim)
            return row + lim;
        row += ml;
        col += ml;
        if (ml < 16)
            break;
    }
    return row;
}

// One extend attempt for U diagonals of a thread at once: the first windows
// of all U are loaded together; a diagonal whose whole window matched goes on
// in extend_run.  A row is in range when 0 <= row < qlen and
// 0 <= row - k < rlen (one unsigned compare each; NEG rows fail).
template <int U, bool SMEM>
__device__ __forceinline__ void extend_u(const SeqHalves &qs, int32_t qlen, const SeqHalves &rs,
                                         int32_t rlen, int32_t (&rows)[U], const int32_t (&ks)[U],
                                         const bool (&live)[U])
{
    uint32_t x[U];
    int32_t lim[U];
    bool go[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t row = rows[u], col = row - ks[u];
        go[u] = live[u] && (uint32_t)row < (uint32_t)qlen && (uint32_t)col < (uint32_t)rlen;
        lim[u] = min(qlen - row, rlen - col);
        x[u] = 0;
        if (go[u])
            x[u] = window16<SMEM>(qs, row) ^ window16<SMEM>(rs, col);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (!go[u])
            continue;
        const int ml = __clz((int)x[u]) >> 1;
        rows[u] += min(ml, lim[u]);
        if (ml == 16 && lim[u] > 16)
            rows[u] = extend_run<SMEM>(qs, qlen, rs, rlen, rows[u], ks[u]);
    }
}

// SMEM: both sequences are copied into shared memory as halves, high half
// first, plus a zero pad word (the caller checked they fit); otherwise both
// are read from their packed words in global memory.
template <int TW, bool SMEM>
__device__ __forceinline__ SeqHalves stage_sequence(const SeqView &v, int64_t off, int32_t nw,
                                                    uint32_t *smem, int tt)
{
    if (SMEM) {
        uint2 *d = reinterpret_cast<uint2 *>(smem);
        for (int i = tt; i <= nw; i += TW) {
            const uint64_t x = i < nw ? __ldg(v.packed + off + i) : 0;
            d[i] = make_uint2((uint32_t)(x >> 32), (uint32_t)x);
        }
        return SeqHalves{smem, 2 * nw, 0u};
    }
    const int64_t last = 2 * (v.n_words - off) - 1;
    return SeqHalves{reinterpret_cast<const uint32_t *>(v.packed + off),
                     (int32_t)min(last, (int64_t)0x7fffffff), 1u};
}

// Pair alignment by a team of TEAM warps (TEAM = 1: one warp; TEAM = 4: the
// whole 128-thread block).  Thread tt of the team owns diagonals
// a + tt + 32*TEAM*j of the visited interval.  Per score step:
//  * ring slots advance by one (no division);
//  * every warp keeps its own copy of the per-slot intervals (lane j holds
//    slot j's) and computes the same [a, b];
//  * the reused destination slots are cleaned only where their old interval
//    pokes out of [a, b];
//  * each thread loads the sources of U diagonals together (they live in
//    other slots than the ones written, so nothing written in the step is
//    read back in it), computes, extends and stores each diagonal once;
//    values below zero are stored as NEG, so NEG never drifts;
//  * the touched interval [GL, GH] is widened at the END of the step, with
//    kWfaWiden spare diagonals, so that it holds [a-2, b+2].  The next
//    step's interval reaches at most one diagonal past every earlier one and
//    reads one more on each side, so its reads stay inside what earlier
//    steps filled, and a step needs one team barrier (which also ORs the
//    "target reached" flags).
// Both sequences are copied into shared memory when both fit seqw - 1 words
// (SMEM); otherwise both are read from global memory.  (seqw counts 64-bit
// words; the copies are stored as 32-bit halves.)
constexpr int kWfaSeqWords = 321;  // per sequence per warp: 10,240 bases + a zero pad
constexpr int kWfaWiden = 30;
constexpr int kWfaTeamSeqWords = 4 * kWfaSeqWords;  // team mode: 41,056 bases + pad

// Team barrier with memory ordering that also ORs a flag over the team.
template <int TEAM>
__device__ __forceinline__ bool team_any(bool v)
{
    if (TEAM == 1) {
        __syncwarp();
        return __any_sync(0xffffffffu, v);
    }
    return __syncthreads_or(v) != 0;
}

template <int TEAM>
__device__ __forceinline__ void team_sync()
{
    if (TEAM == 1)
        __syncwarp();
    else
        __syncthreads();
}

struct WfaShape {
    int g, xs, oes, es, hm, hie, nslot;
};

// Ring element: int32 (NEG = -2^30) or int16 (NEG = -32768): half the ring
// bytes.  A value gains at most one per score step, so after S steps rows are
// at most qlen + S and a value that started at NEG is at most NEG + S.  The
// int16 path runs only while S <= 32767 - qlen, where rows fit and
// NEG + S <= -1 - qlen stays negative -- so negative values need no
// renormalisation there; a pair that needs more steps returns -4 and is run
// again with int32 rings.  The int32 path stores every negative result as
// NEG.  Arithmetic is int32 either way.
template <typename RT> struct RingNeg;
template <> struct RingNeg<int32_t> {
    static constexpr int32_t value = WFA_NEG;
};
template <> struct RingNeg<int16_t> {
    static constexpr int32_t value = -32768;
};

// HREC: also write the pair's history record (the CIGAR pass): at most
// hsteps score indices (the cost is known), into hrec, whose cell part ends
// at 4-byte word hlimit; a step that would pass it makes the call return -3.
// Returns the cost (team-uniform).
template <int U, int TEAM, bool SMEM, typename RT, bool HREC>
__device__ __forceinline__ int32_t wfa_align_pair(const SeqView &q, const SeqView &r,
                                                  const WfaParams &p, const WfaShape &w,
                                                  int64_t pi, int32_t *region, int64_t slot_width,
                                                  uint32_t *sq, uint32_t *sr,
                                                  int32_t *__restrict__ out, int *err_flag,
                                                  int64_t *work, int64_t *hist, uint8_t *hrec,
                                                  int64_t hlimit, int hsteps)
{
    constexpr int TW = TEAM * 32;
    constexpr int32_t NEG = RingNeg<RT>::value;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tt = TEAM == 1 ? lane : (int)threadIdx.x;
    const int hm = w.hm, hie = w.hie, xs = w.xs, oes = w.oes, es = w.es, g = w.g;
    const int32_t max_err = p.max_error;
    const int64_t qoff = q.offsets[pi] - q.word_base;
    const int64_t roff = r.offsets[pi] - r.word_base;
    const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
    int32_t result = -1;
    int64_t cells = 0;
    int64_t hbytes = 8;  // history bytes of the visited cells (score 0: one cell)
    int32_t *const hdr = reinterpret_cast<int32_t *>(hrec);
    int64_t hcur = 3 * (int64_t)hsteps;  // next free 4-byte word of the record
    bool overrun = false, need32 = false;
    const int64_t ql64 = q.lengths[pi], rl64 = r.lengths[pi];
    if (ql64 < 0 || rl64 < 0 || ql64 + rl64 + 5 > slot_width) {
        // a length the caller's bounds did not cover (negative, 2^31 or more, or
        // past the rings): cost -2 and the error flag
        if (tt == 0)
            atomicOr(err_flag, 1);
        result = -2;
    } else if (qlen == 0 && rlen == 0) {
        result = 0;
    } else if ((int64_t)qlen + rlen + 5 > slot_width) {
        if (tt == 0)
            atomicOr(err_flag, 1);
        result = -2;
    } else {
        const int32_t qnw = (qlen + 31) >> 5, rnw = (rlen + 31) >> 5;
        team_sync<TEAM>();  // the previous pair's reads of the shared copies are done
        const SeqHalves qs = stage_sequence<TW, SMEM>(q, qoff, qnw, sq, tt);
        const SeqHalves rs = stage_sequence<TW, SMEM>(r, roff, rnw, sr, tt);
        const int32_t kofs = rlen + 2;
        const int32_t target = qlen - rlen;
        RT *const base = reinterpret_cast<RT *>(region) + kofs;
        auto M = [&](int slot) { return base + (int64_t)slot * slot_width; };
        auto I = [&](int slot) { return base + (int64_t)(hm + slot) * slot_width; };
        auto D = [&](int slot) { return base + (int64_t)(hm + hie + slot) * slot_width; };
        // per-slot intervals: lane j holds M slot j's and I/D slot j's (I and
        // D of one score always share their interval; ring sizes <= 32)
        int32_t mlo = 1, mhi = 0, ilo = 1, ihi = 0;
        int32_t GL = max(-2, -rlen - 2), GH = min(2, qlen + 2);
        for (int sl = 0; sl < w.nslot; ++sl) {
            RT *row = base + (int64_t)sl * slot_width;
            for (int32_t k = GL + tt; k <= GH; k += TW)
                row[k] = NEG;
        }
        team_sync<TEAM>();
        // score 0: M[0,0] = 0 extended along diagonal 0 (:130-140); every
        // thread computes it, thread 0 stores it
        const int32_t row0 = extend_run<SMEM>(qs, qlen, rs, rlen, 0, 0);
        if (lane == 0) {
            mlo = 0;
            mhi = 0;
        }
        if (tt == 0)
            M(0)[0] = (RT)row0;
        if (HREC) {
            if (tt == 0) {
                hdr[0] = 0;
                hdr[1] = 0;
                hdr[2] = (int32_t)hcur;
                hdr[hcur] = row0;
                hrec[(hcur + 1) * 4] = 0;
            }
            hcur += wfa_hist_cell_bytes(1) / 4;
        }
        team_sync<TEAM>();
        if (target == 0 && row0 >= qlen) {
            result = 0;
        } else {
            int ms = 0, is = 0;  // ring slots of the current score
            for (int64_t sp = 1; HREC ? sp < hsteps : sp * g <= max_err; ++sp) {
                if (std::is_same<RT, int16_t>::value && sp > 32767 - (int64_t)qlen) {
                    need32 = true;  // past the steps int16 values are proven for
                    break;
                }
                const int32_t s = (int32_t)(sp * g);
                ms = ms + 1 == hm ? 0 : ms + 1;
                is = is + 1 == hie ? 0 : is + 1;
                int32_t lo = max(-rlen, -s), hi = min(qlen, s);
                if (target < lo || target > hi) {
                    lo = min(lo, target);
                    hi = max(hi, target);
                }
                lo = max(lo, -max_err);
                hi = min(hi, max_err);
                const int sx = sp >= xs ? (ms >= xs ? ms - xs : ms - xs + hm) : -1;
                const int soe = sp >= oes ? (ms >= oes ? ms - oes : ms - oes + hm) : -1;
                const int se = sp >= es ? (is >= es ? is - es : is - es + hie) : -1;
                int32_t ulo = 0x7fffffff, uhi = -0x7fffffff;
                {
                    const int32_t a0 = __shfl_sync(FULL, mlo, sx & 31);
                    const int32_t b0 = __shfl_sync(FULL, mhi, sx & 31);
                    if (sx >= 0 && a0 <= b0) {
                        ulo = a0;
                        uhi = b0;
                    }
                    const int32_t a1 = __shfl_sync(FULL, mlo, soe & 31);
                    const int32_t b1 = __shfl_sync(FULL, mhi, soe & 31);
                    if (soe >= 0 && a1 <= b1) {
                        ulo = min(ulo, a1 - 1);
                        uhi = max(uhi, b1 + 1);
                    }
                    const int32_t a2 = __shfl_sync(FULL, ilo, se & 31);
                    const int32_t b2 = __shfl_sync(FULL, ihi, se & 31);
                    if (se >= 0 && a2 <= b2) {  // I[s-e] at k-1 and D[s-e] at k+1
                        ulo = min(ulo, a2 - 1);
                        uhi = max(uhi, b2 + 1);
                    }
                }
                const int32_t a = max(ulo, lo);
                const int32_t b = min(uhi, hi);
                const int32_t omlo = __shfl_sync(FULL, mlo, ms);
                const int32_t omhi = __shfl_sync(FULL, mhi, ms);
                const int32_t oilo = __shfl_sync(FULL, ilo, is);
                const int32_t oihi = __shfl_sync(FULL, ihi, is);
                RT *const Mw = M(ms), *const Iw = I(is), *const Dw = D(is);
                // what the reused slots held outside [a, b] becomes NEG (all
                // of it when this score is empty)
                const int32_t ca = a > b ? 0x7fffffff : a, cb = a > b ? -0x7fffffff : b;
                if ((omlo <= omhi && (omlo < ca || omhi > cb)) ||
                    (oilo <= oihi && (oilo < ca || oihi > cb))) {
                    for (int32_t k = omlo + tt; k <= min(omhi, ca - 1); k += TW)
                        Mw[k] = NEG;
                    for (int32_t k = max(omlo, cb + 1) + tt; k <= omhi; k += TW)
                        Mw[k] = NEG;
                    for (int32_t k = oilo + tt; k <= min(oihi, ca - 1); k += TW) {
                        Iw[k] = NEG;
                        Dw[k] = NEG;
                    }
                    for (int32_t k = max(oilo, cb + 1) + tt; k <= oihi; k += TW) {
                        Iw[k] = NEG;
                        Dw[k] = NEG;
                    }
                }
                int32_t *hm_out = nullptr;  // this score's part of the record
                uint8_t *hd_out = nullptr;
                if (HREC) {
                    if (a <= b && hcur + wfa_hist_cell_bytes(b - a + 1) / 4 > hlimit) {
                        overrun = true;  // same decision in every thread
                        break;
                    }
                    if (tt == 0) {
                        hdr[3 * sp] = a <= b ? a : 1;
                        hdr[3 * sp + 1] = a <= b ? b : 0;
                        hdr[3 * sp + 2] = a <= b ? (int32_t)hcur : 0;
                    }
                    hm_out = hdr + hcur;
                    hd_out = hrec + (hcur + (b - a + 1)) * 4;
                }
                bool hit = false;
                if (a <= b) {
                    cells += (int64_t)(b - a + 1);
                    hbytes += wfa_hist_cell_bytes(b - a + 1);
                    const RT *Mx = sx >= 0 ? M(sx) : nullptr;
                    const RT *Moe = soe >= 0 ? M(soe) : nullptr;
                    const RT *Ie = se >= 0 ? I(se) : nullptr;
                    const RT *De = se >= 0 ? D(se) : nullptr;
                    // rounds of U diagonals per thread while all U are inside
                    // [a, b], then single-diagonal rounds for the rest
                    // FULL: every diagonal of the round lies inside [a, b] (no
                    // liveness tests, addresses linear in u)
                    auto round = [&](int32_t k0, auto uc, auto fc) {
                        constexpr int UU = decltype(uc)::value;
                        constexpr bool FULL = decltype(fc)::value;
                        int32_t ks[UU], iv[UU], dv[UU], mv[UU];
                        uint32_t dec[UU];
                        bool live[UU];
#pragma unroll
                        for (int u = 0; u < UU; ++u) {
                            ks[u] = k0 + TW * u;
                            live[u] = FULL || ks[u] <= b;
                            // loads stay in [a-1, b+1]
                            const int32_t kc = FULL ? ks[u] : (live[u] ? ks[u] : b);
                            int32_t io = NEG, ie = NEG, dop = NEG, dex = NEG, mx = NEG;
                            if (Moe) {
                                io = (int32_t)Moe[kc - 1];
                                dop = (int32_t)Moe[kc + 1];
                            }
                            if (Ie) {
                                ie = (int32_t)Ie[kc - 1];
                                dex = (int32_t)De[kc + 1];
                            }
                            if (Mx)
                                mx = (int32_t)Mx[kc];
                            const int32_t i0 = max(io, ie), d0 = max(dop, dex), m0 = mx + 1;
                            // max(mx + 1, i0 + 1, d0) as two DPX add-max instructions
                            const int32_t m1 = __viaddmax_s32(mx, 1, __viaddmax_s32(i0, 1, d0));
                            if (HREC) {
                                // the traceback's tests (align_cpu.mojo:509-601), first
                                // equal source: M from mismatch, I, D; I / D from an
                                // open before an extension
                                uint32_t d = 0;
                                if (m1 >= 0)
                                    d = (mx >= 0 && m0 == m1) ? 1u
                                                              : ((i0 >= 0 && i0 + 1 == m1) ? 2u : 3u);
                                if (i0 >= 0 && !(io >= 0 && io == i0))
                                    d |= 4u;
                                if (d0 >= 0 && !(dop >= 0 && dop == d0))
                                    d |= 8u;
                                dec[u] = d;
                            }
                            if (std::is_same<RT, int16_t>::value) {
                                iv[u] = i0 + 1;
                                mv[u] = m1;
                            } else {
                                iv[u] = i0 < 0 ? NEG : i0 + 1;
                                mv[u] = m1 < 0 ? NEG : m1;
                            }
                            dv[u] = d0;
                        }
                        extend_u<UU, SMEM>(qs, qlen, rs, rlen, mv, ks, live);
#pragma unroll
                        for (int u = 0; u < UU; ++u) {
                            if (live[u]) {
                                Iw[ks[u]] = (RT)iv[u];
                                Dw[ks[u]] = (RT)dv[u];
                                Mw[ks[u]] = (RT)mv[u];
                                if (HREC) {
                                    hm_out[ks[u] - a] = mv[u];
                                    hd_out[ks[u] - a] = (uint8_t)dec[u];
                                }
                            }
                        }
                    };
                    int32_t k0 = a + tt;
                    for (; k0 + TW * (U - 1) <= b; k0 += TW * U)
                        round(k0, std::integral_constant<int, U>{}, std::true_type{});
                    for (; k0 <= b; k0 += TW)
                        round(k0, std::integral_constant<int, 1>{}, std::false_type{});
                    // the thread that owns the target diagonal reads back what it
                    // stored there this step (its own store, so program order holds)
                    if (target >= a && target <= b && ((target - a) & (TW - 1)) == tt)
                        hit = (int32_t)Mw[target] >= qlen;
                    if (HREC)
                        hcur += wfa_hist_cell_bytes(b - a + 1) / 4;
                    // widen for the next step (see above); the positions
                    // filled lie outside everything this step reads or writes
                    if (a - 2 < GL || b + 2 > GH) {
                        const int32_t nGL = a - 2 < GL ? max(a - 2 - kWfaWiden, -rlen - 2) : GL;
                        const int32_t nGH = b + 2 > GH ? min(b + 2 + kWfaWiden, qlen + 2) : GH;
                        for (int sl = 0; sl < w.nslot; ++sl) {
                            RT *rowp = base + (int64_t)sl * slot_width;
                            for (int32_t k = nGL + tt; k < GL; k += TW)
                                rowp[k] = NEG;
                            for (int32_t k = GH + 1 + tt; k <= nGH; k += TW)
                                rowp[k] = NEG;
                        }
                        GL = nGL;
                        GH = nGH;
                    }
                }
                if (lane == ms) {
                    mlo = a <= b ? a : 1;
                    mhi = a <= b ? b : 0;
                }
                if (lane == is) {
                    ilo = a <= b ? a : 1;
                    ihi = a <= b ? b : 0;
                }
                // M[s, target] >= qlen ends the alignment (:221-224); target
                // inside [a, b] is inside the reference's [lo, hi]
                if (team_any<TEAM>(hit)) {
                    result = s;
                    break;
                }
            }
        }
    }
    if (need32)
        return -4;  // nothing written: the caller runs the pair with int32 rings
    if (tt == 0) {
        if (out)
            out[pi] = result;
        if (work)
            atomicAdd((unsigned long long *)work, (unsigned long long)cells);
        if (hist)
            hist[pi] = result >= 0 ? hbytes : 0;
    }
    return overrun ? -3 : result;
}

// Runs pair pi with the shared-memory copies when both sequences fit seqw
// words (with the pad) and with int16 rings when its rows fit them.
template <int U, int TEAM, bool HREC = false>
__device__ __forceinline__ int32_t wfa_pair_dispatch(const SeqView &q, const SeqView &r,
                                                     const WfaParams &p, const WfaShape &w,
                                                     int64_t pi, int32_t *region,
                                                     int64_t slot_width, uint32_t *sq,
                                                     uint32_t *sr, int seqw, int32_t *out,
                                                     int *err_flag, int64_t *work, int64_t *hist,
                                                     uint8_t *hrec = nullptr, int64_t hlimit = 0,
                                                     int hsteps = 0)
{
    const int64_t ql = q.lengths[pi], rl = r.lengths[pi];
    const bool smem = ((ql + 31) >> 5) < seqw && ((rl + 31) >> 5) < seqw;
    const bool r16 = ql < 32767;
    int32_t res = -4;
    if (smem) {
        if (r16)
            res = wfa_align_pair<U, TEAM, true, int16_t, HREC>(q, r, p, w, pi, region, slot_width,
                                                               sq, sr, out, err_flag, work, hist,
                                                               hrec, hlimit, hsteps);
        if (res == -4)
            res = wfa_align_pair<U, TEAM, true, int32_t, HREC>(q, r, p, w, pi, region, slot_width,
                                                               sq, sr, out, err_flag, work, hist,
                                                               hrec, hlimit, hsteps);
        return res;
    }
    if (r16)
        res = wfa_align_pair<U, TEAM, false, int16_t, HREC>(q, r, p, w, pi, region, slot_width,
                                                            sq, sr, out, err_flag, work, hist,
                                                            hrec, hlimit, hsteps);
    if (res == -4)
        res = wfa_align_pair<U, TEAM, false, int32_t, HREC>(q, r, p, w, pi, region, slot_width,
                                                            sq, sr, out, err_flag, work, hist,
                                                            hrec, hlimit, hsteps);
    return res;
}

// Persistent kernel over two length-sorted queues: every block first takes
// pairs of `longs` one at a time as a team of its BW warps (a long pair's
// score steps are its critical path, so the block's warps share each step);
// when that queue is empty each warp takes pairs of `shorts` on its own.  Ring
// slots: one region of nslot * slot_width int32 per warp (team mode uses the
// block's first).  Shared memory (dynamic): per warp two sequence copies of
// kWfaSeqWords words, BW * 4 * kWfaSeqWords uint32 in all.
// BW = 4: five resident blocks per SM (96 registers, no spills) beat four with
// more registers; six or more spill and run slower.  BW = 16: one 512-thread
// block per SM, so each of the longest pairs gets a whole SM's 16 warps.
template <int U, int BW>
__global__ void __launch_bounds__(32 * BW, BW == 4 ? 5 : 1)
wfa_kernel(SeqView q, SeqView r, WfaParams p, PairList longs, PairList shorts,
           int32_t *__restrict__ out, int32_t *__restrict__ scratch, int64_t slot_width,
           int *err_flag, int64_t *work, int64_t *hist)
{
    static_assert(BW >= 4, "team copies need 4 warps' share of shared memory");
    extern __shared__ __align__(16) uint32_t seqs[];
    __shared__ int64_t team_slot;
    WfaShape w;
    w.g = gcd_i(p.x, gcd_i(p.o, p.e));
    w.xs = p.x / w.g;
    w.oes = (p.o + p.e) / w.g;
    w.es = p.e / w.g;
    w.hm = max(w.xs, w.oes) + 1;
    w.hie = w.es + 1;
    w.nslot = w.hm + 2 * w.hie;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t region_words = (int64_t)w.nslot * slot_width;

    int64_t nl;
    const int32_t *__restrict__ lq = pairs_resolve(longs, nl);
    if (nl > 0) {
        int32_t *const region = scratch + (int64_t)blockIdx.x * BW * region_words;
        for (;;) {
            __syncthreads();
            if (threadIdx.x == 0)
                team_slot = atomicAdd(longs.counter, 1);
            __syncthreads();
            const int64_t si = team_slot;
            if (si >= nl)
                break;
            const int64_t pi = lq ? (int64_t)lq[si] : si;
            wfa_pair_dispatch<U, BW>(q, r, p, w, pi, region, slot_width, seqs,
                                    seqs + 2 * kWfaTeamSeqWords, kWfaTeamSeqWords, out, err_flag,
                                    work, hist);
        }
        __syncthreads();  // shared copies of the last long pair are no longer read
    }

    int64_t ns;
    const int32_t *__restrict__ sq = pairs_resolve(shorts, ns);
    int32_t *const region = scratch + ((int64_t)blockIdx.x * BW + wib) * region_words;
    uint32_t *const my = seqs + wib * 4 * kWfaSeqWords;
    for (;;) {
        int64_t b0 = 0;
        if (lane == 0)
            b0 = atomicAdd(shorts.counter, 1);
        const int64_t si = __shfl_sync(0xffffffffu, b0, 0);
        if (si >= ns)
            break;
        const int64_t pi = sq ? (int64_t)sq[si] : si;
        wfa_pair_dispatch<U, 1>(q, r, p, w, pi, region, slot_width, my, my + 2 * kWfaSeqWords,
                                kWfaSeqWords, out, err_flag, work, hist);
    }
}

// CIGAR pass (see wfa_cigar.cu): re-runs the forward pass of pairs whose cost
// is known with wfa_align_pair in history mode, then one thread walks the
// record back into runs.  The first n_team pairs of the list (the largest
// records) are taken one per block by its 4 warps, the rest one per warp, as
// in wfa_kernel.
template <int TEAM>
__device__ __forceinline__ void cigar_pair(const SeqView &q, const SeqView &r, const WfaParams &p,
                                           const WfaShape &w, int64_t pi, int32_t *region,
                                           int64_t slot_width, uint32_t *sq, uint32_t *sr,
                                           int seqw, const int32_t *cost,
                                           const int64_t *hist_cells, const int64_t *arena_off,
                                           uint8_t *arena, uint32_t *runs,
                                           const int64_t *run_off, int32_t *run_count,
                                           int *err_flag)
{
    const int tt = TEAM == 1 ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
    const int32_t c = cost[pi];
    const int64_t qlen = q.lengths[pi], rlen = r.lengths[pi];
    if (c < 0 || (qlen == 0 && rlen == 0)) {
        if (tt == 0)
            run_count[pi] = 0;
        return;
    }
    if (qlen + rlen + 5 > slot_width || c % w.g != 0) {
        if (tt == 0) {
            atomicOr(err_flag, 1);
            run_count[pi] = -1;
        }
        return;
    }
    const int S = c / w.g + 1;
    uint8_t *const rec = arena + arena_off[pi];
    const int64_t limit = 3 * (int64_t)S + hist_cells[pi] / 4;
    const int32_t res = wfa_pair_dispatch<4, TEAM, true>(q, r, p, w, pi, region, slot_width, sq,
                                                         sr, seqw, nullptr, err_flag, nullptr,
                                                         nullptr, rec, limit, S);
    team_sync<TEAM>();  // the record is complete and visible to thread 0
    if (tt != 0)
        return;
    if (res != c) {  // the cost pass and this pass disagree
        atomicOr(err_flag, 2);
        run_count[pi] = -1;
        return;
    }
    const int64_t nrun = wfa_traceback(rec, c, w.g, w.xs, w.oes, w.es, (int32_t)qlen,
                                       (int32_t)rlen, runs + run_off[pi], qlen + rlen + 1);
    if (nrun < 0) {
        atomicOr(err_flag, 4);
        run_count[pi] = -1;
    } else {
        run_count[pi] = (int32_t)nrun;
    }
}

__global__ void __launch_bounds__(128)
wfa_cigar_kernel(SeqView q, SeqView r, WfaParams p, const int32_t *__restrict__ pairs, int64_t n,
                 int64_t n_team, int *counters, const int32_t *__restrict__ cost,
                 const int64_t *__restrict__ hist_cells, const int64_t *__restrict__ arena_off,
                 uint8_t *__restrict__ arena, int32_t *__restrict__ scratch, int64_t slot_width,
                 uint32_t *__restrict__ runs, const int64_t *__restrict__ run_off,
                 int32_t *__restrict__ run_count, int *err_flag)
{
    __shared__ __align__(16) uint32_t seqs[4 * 2 * 2 * kWfaSeqWords];
    __shared__ int64_t team_slot;
    WfaShape w;
    w.g = gcd_i(p.x, gcd_i(p.o, p.e));
    w.xs = p.x / w.g;
    w.oes = (p.o + p.e) / w.g;
    w.es = p.e / w.g;
    w.hm = max(w.xs, w.oes) + 1;
    w.hie = w.es + 1;
    w.nslot = w.hm + 2 * w.hie;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t region_words = (int64_t)w.nslot * slot_width;
    if (n_team > 0) {
        int32_t *const region = scratch + (int64_t)blockIdx.x * 4 * region_words;
        for (;;) {
            __syncthreads();
            if (threadIdx.x == 0)
                team_slot = atomicAdd(counters + 32, 1);
            __syncthreads();
            const int64_t si = team_slot;
            if (si >= n_team)
                break;
            cigar_pair<4>(q, r, p, w, pairs[si], region, slot_width, seqs,
                          seqs + 2 * kWfaTeamSeqWords, kWfaTeamSeqWords, cost, hist_cells,
                          arena_off, arena, runs, run_off, run_count, err_flag);
        }
        __syncthreads();
    }
    int32_t *const region = scratch + ((int64_t)blockIdx.x * 4 + wib) * region_words;
    uint32_t *const my = seqs + wib * 4 * kWfaSeqWords;
    for (;;) {
        int64_t b0 = 0;
        if (lane == 0)
            b0 = n_team + atomicAdd(counters, 1);
        const int64_t si = __shfl_sync(0xffffffffu, b0, 0);
        if (si >= n)
            break;
        cigar_pair<1>(q, r, p, w, pairs[si], region, slot_width, my, my + 2 * kWfaSeqWords,
                      kWfaSeqWords, cost, hist_cells, arena_off, arena, runs, run_off,
                      run_count, err_flag);
    }
}

cudaError_t launch_wfa_cigar(SeqView q, SeqView r, WfaParams p, const int32_t *pairs, int64_t n,
                             int64_t n_team, int *counters, const int32_t *cost,
                             const int64_t *hist_cells, const int64_t *arena_off, uint8_t *arena,
                             int32_t *scratch, int64_t slot_width, int grid, uint32_t *runs,
                             const int64_t *run_off, int32_t *run_count, int *err_flag,
                             cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    wfa_cigar_kernel<<<grid, 128, 0, st>>>(q, r, p, pairs, n, n_team, counters, cost,
                                           hist_cells, arena_off, arena, scratch, slot_width, runs,
                                           run_off, run_count, err_flag);
    return cudaGetLastError();
}

int wfa_cigar_blocks_per_sm()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, wfa_cigar_kernel, 128, 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    return nb > 0 ? nb : 1;
}

static size_t wfa_smem_bytes(int bw) { return (size_t)bw * 4 * kWfaSeqWords * 4; }

// One-time opt-in to the kernel's dynamic shared memory (above 48 KB for BW = 16).
template <int U, int BW>
static void wfa_prepare()
{
    static const cudaError_t e = cudaFuncSetAttribute(
        wfa_kernel<U, BW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wfa_smem_bytes(BW));
    (void)e;
}

template <int U, int BW>
static int wfa_occupancy()
{
    wfa_prepare<U, BW>();
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wfa_kernel<U, BW>, 32 * BW,
                                                      wfa_smem_bytes(BW)) != cudaSuccess) {
        cudaGetLastError();
        return BW == 4 ? 4 : 1;
    }
    return n > 0 ? n : 1;
}

int wfa_blocks_per_sm(int variant, int block_warps)
{
    if (block_warps == kWfaWideWarps)
        return wfa_occupancy<4, kWfaWideWarps>();
    if (variant & 0x20)
        return wfa_occupancy<1, 4>();
    if (variant & 0x10)
        return wfa_occupancy<2, 4>();
    return wfa_occupancy<4, 4>();
}

cudaError_t launch_wfa(int variant, int block_warps, SeqView q, SeqView r, WfaParams p,
                       PairList longs, PairList shorts, int32_t *out, int32_t *scratch,
                       int64_t slot_width, int grid, int *err_flag, int64_t *work, int64_t *hist,
                       cudaStream_t st)
{
    // block_warps kWfaWideWarps: the wide kernel (4 diagonals per thread per
    // round); otherwise variant bits 4-5: diagonals per thread per round 4
    // (default), 2 or 1
    if (block_warps == kWfaWideWarps) {
        wfa_prepare<4, kWfaWideWarps>();
        wfa_kernel<4, kWfaWideWarps><<<grid, 32 * kWfaWideWarps, wfa_smem_bytes(kWfaWideWarps),
                                       st>>>(q, r, p, longs, shorts, out, scratch, slot_width,
                                             err_flag, work, hist);
    } else if (variant & 0x20) {
        wfa_prepare<1, 4>();
        wfa_kernel<1, 4><<<grid, 128, wfa_smem_bytes(4), st>>>(
            q, r, p, longs, shorts, out, scratch, slot_width, err_flag, work, hist);
    } else if (variant & 0x10) {
        wfa_prepare<2, 4>();
        wfa_kernel<2, 4><<<grid, 128, wfa_smem_bytes(4), st>>>(
            q, r, p, longs, shorts, out, scratch, slot_width, err_flag, work, hist);
    } else {
        wfa_prepare<4, 4>();
        wfa_kernel<4, 4><<<grid, 128, wfa_smem_bytes(4), st>>>(
            q, r, p, longs, shorts, out, scratch, slot_width, err_flag, work, hist);
    }
    return cudaGetLastError();
}

// ---- integer throughput probe -------------------------------------------------
// Eight independent chains per thread of one operation class; the result is
// stored so the chains cannot be removed.
__global__ void int_peak_kernel(int kind, int iters, uint32_t *sink)
{
    uint32_t a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        a[i] = threadIdx.x * 2654435761u + i * 40503u + blockIdx.x;
    const uint32_t c1 = sink[1] | 3u, c2 = sink[2] | 5u;
    switch (kind) {
    case 0:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = a[i] + a[(i + 1) & 7] + c1;
        break;
    case 1:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = (uint32_t)max((int32_t)a[i], (int32_t)a[(i + 3) & 7]);
        break;
    case 2:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = (uint32_t)__viaddmax_s32((int32_t)a[i], (int32_t)c1, (int32_t)a[(i + 1) & 7]);
        break;
    case 3:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __viaddmax_s16x2(a[i], c1, a[(i + 1) & 7]);
        break;
    case 4:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = (uint32_t)__vimax3_s32((int32_t)a[i], (int32_t)a[(i + 1) & 7],
                                              (int32_t)a[(i + 2) & 7]);
        break;
    case 5:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = (a[i] & a[(i + 1) & 7]) ^ c2;
        break;
    case 6:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = a[i] * c1 + a[(i + 1) & 7];
        break;
    case 7:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __shfl_xor_sync(0xffffffffu, a[i], 1) + c1;
        break;
    case 8:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __vimax3_s16x2(a[i], a[(i + 1) & 7], a[(i + 2) & 7]);
        break;
    case 9:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __vimax3_u16x2(a[i], a[(i + 1) & 7], a[(i + 2) & 7]);
        break;
    case 10:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __byte_perm(a[i], a[(i + 1) & 7], 0x7632);
        break;
    case 11:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __viaddmax_s16x2_relu(a[i], c1, a[(i + 1) & 7]);
        break;
    default:
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a[i] = __vimax_s16x2_relu(a[i], a[(i + 1) & 7]);
        break;
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        s ^= a[i];
    if (s == 0x9E3779B9u)
        sink[0] = s;
}

cudaError_t launch_int_peak(int kind, int grid, int block, int iters, uint32_t *sink,
                            cudaStream_t st)
{
    int_peak_kernel<<<grid, block, 0, st>>>(kind, iters, sink);
    return cudaGetLastError();
}

}  // namespace gb2
