// wfa_tiers.cu -- gap-affine WFA cost with the wavefront rings in shared memory.
//
// Computes wfa_affine_cpu (genomics/cpu/align_cpu.mojo:75-226) exactly, with
// the recurrences, equivalences and termination of wfa_kernels.cu (see its
// header): scores visited in steps of g = gcd(x, o, e), only the diagonals
// the sources reach, intersected with the reference's [lo, hi] (:158-164),
// negative values stored as NEG.
//
// Storage.  A pair's M/I/D rings (nslot = hm + 2*hie slots, 9 for x4 o6 e2)
// live in a window of W int16 elements per slot, diagonal k at element
// H + k.  The visited interval after S steps lies inside [-S, S] (a source
// reaches one diagonal further per step), so the window fills from its
// centre outwards and every element is NEG-filled once when the pair starts;
// afterwards each step only overwrites its own interval and turns what the
// reused slot held outside it back into NEG.  Reads at k-1 and k+1 therefore
// need no bounds tests, and the neighbours of a diagonal are fixed offsets.
//
// Tiers.  Work per pair grows with the square of its cost (most pairs are
// cheap, most cells are in the few expensive ones), so a pair starts on the
// smallest team and moves up when its interval outgrows the window:
//   T1   one warp per pair,      sixteen per block, W = 616  (x4 o6 e2)
//   T2   two warps per pair,     eight per block,   W = 1,240
//   T4   four warps per pair,    four per block,    W = 2,488
//   T8   eight warps per pair,   two per block,     W = 4,984
//   T16  sixteen warps per pair, one per block,     W = 9,968
// each in its own launch, one after another on the executor's stream.  A
// pair whose next step would read or write outside its window is suspended:
// the team writes its state (slot intervals, step, ring contents over the
// live span) to a dump record in HBM and queues the pair for the next tier,
// whose launch restores it into its larger window and continues from the
// same step.  No cell is computed twice.  A pair that outgrows T16, or whose
// rows could leave int16 (qlen + steps > 32767), runs from the start in the
// G tier: sixteen warps per pair with int32 rings in a per-block region of
// global memory large enough for any interval ([-max(qlen, rlen) - 3, ...]).
// When the dump space of a transition is used up, the pair starts over in
// the next tier instead (same results, more work).
//
// Sequences are copied into shared memory as overlapping 64-bit windows
// (entry j = 16-base halves j and j+1), so a 16-base window at any position
// is one 64-bit load and one funnel shift; pairs longer than a tier's copy
// capacity read their windows from the packed words in global memory.
#include <type_traits>

#include "gb2_internal.cuh"

namespace gb2 {
namespace {

constexpr int32_t kPromote = -10;  // suspended: the pair continues in the next tier
constexpr int32_t kRestart = -11;  // must start over in the G tier (int32 rings)
constexpr int32_t kRunning = -12;  // internal: no result yet
constexpr int kDumpHeader = 1024;  // bytes of a dump record before the ring data

struct Shape {
    int g, xs, oes, es, hm, hie, nslot;
};

__device__ __forceinline__ int gcd_d(int a, int b)
{
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

__device__ __forceinline__ Shape make_shape(const WfaParams &p)
{
    Shape w;
    w.g = gcd_d(p.x, gcd_d(p.o, p.e));
    w.xs = p.x / w.g;
    w.oes = (p.o + p.e) / w.g;
    w.es = p.e / w.g;
    w.hm = max(w.xs, w.oes) + 1;
    w.hie = w.es + 1;
    w.nslot = w.hm + 2 * w.hie;
    return w;
}

template <typename RT> struct Neg;
template <> struct Neg<int16_t> {
    static constexpr int32_t value = -32768;
};
template <> struct Neg<int32_t> {
    static constexpr int32_t value = -(1 << 30);
};

// ---- team synchronisation ----------------------------------------------------
// TEAM warps align one pair; a block holds NTEAMS teams.  A whole block uses
// __syncthreads, a part of a block a named barrier (id 1 + team), a warp
// __syncwarp.  Both forms order shared and global memory among the team.
template <int TEAM, int NTEAMS>
struct Team {
    int id;  // team index in the block
    __device__ __forceinline__ void sync() const
    {
        if (TEAM == 1)
            __syncwarp();
        else if (NTEAMS == 1)
            __syncthreads();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(1 + id), "r"(TEAM * 32) : "memory");
    }
    // barrier that also ORs v over the team
    __device__ __forceinline__ bool any(bool v) const
    {
        if (TEAM == 1) {
            __syncwarp();
            return __any_sync(0xffffffffu, v);
        }
        if (NTEAMS == 1)
            return __syncthreads_or(v) != 0;
        uint32_t res;
        asm volatile(
            "{\n\t.reg .pred pi, po;\n\t"
            "setp.ne.u32 pi, %1, 0;\n\t"
            "bar.red.or.pred po, %2, %3, pi;\n\t"
            "selp.u32 %0, 1, 0, po;\n\t}"
            : "=r"(res)
            : "r"((uint32_t)v), "r"(1 + id), "r"(TEAM * 32)
            : "memory");
        return res != 0;
    }
};

// ---- sequences ---------------------------------------------------------------
// 16-base windows of a sequence: from the shared copy (win[j] = {half j, half
// j+1}, halves MSB-first) or from the packed little-endian words in global
// memory (logical half j at 32-bit index j ^ 1, clamped to the array).
struct SeqWin {
    const uint2 *win;
    const uint32_t *w32;
    int32_t last;
};

template <bool SMEM>
__device__ __forceinline__ uint32_t win16(const SeqWin &s, int32_t pos)
{
    const int32_t j = pos >> 4;
    if (SMEM) {
        const uint2 e = s.win[j];
        return __funnelshift_l(e.y, e.x, (uint32_t)pos << 1);
    }
    const uint32_t hi = __ldg(s.w32 + ((uint32_t)j ^ 1u));
    const uint32_t lo = __ldg(s.w32 + ((uint32_t)min(j + 1, s.last) ^ 1u));
    return __funnelshift_l(lo, hi, (uint32_t)pos << 1);
}

// Copies nw packed words (2*nw halves) into win[0 .. 2*nw) when SMEM.
template <bool SMEM>
__device__ __forceinline__ SeqWin stage_seq(const SeqView &v, int64_t off, int32_t nw, uint2 *win,
                                            int tt, int tw)
{
    if (SMEM) {
        const int32_t nh = 2 * nw;
        const uint64_t *src = v.packed + off;
        for (int32_t i = tt; i < nh; i += tw) {
            const uint64_t a = __ldg(src + (i >> 1));
            const uint32_t hj = (i & 1) ? (uint32_t)a : (uint32_t)(a >> 32);
            uint32_t hj1 = 0;
            if (i + 1 < nh) {
                const uint64_t b = __ldg(src + ((i + 1) >> 1));
                hj1 = ((i + 1) & 1) ? (uint32_t)b : (uint32_t)(b >> 32);
            }
            win[i] = make_uint2(hj, hj1);
        }
        return SeqWin{win, nullptr, 0};
    }
    const int64_t last = 2 * (v.n_words - off) - 1;
    return SeqWin{nullptr, reinterpret_cast<const uint32_t *>(v.packed + off),
                  (int32_t)min(last, (int64_t)0x7fffffff)};
}

// Extend along diagonal k from row (align_cpu.mojo:208-219): XOR of the two
// 16-base windows, leading zeros / 2 = matching bases, clamped by the
// remaining lengths.  Requires row >= 0 and row - k >= 0.
template <bool SMEM>
__device__ __noinline__ int32_t ext_run(const SeqWin &qs, int32_t qlen, const SeqWin &rs,
                                           int32_t rlen, int32_t row, int32_t k)
{
    int32_t col = row - k;
    while (row < qlen && col < rlen) {
        const uint32_t x = win16<SMEM>(qs, row) ^ win16<SMEM>(rs, col);
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

// First window of U diagonals at once; the ones whose whole window matched
// go on one by one.  In range: 0 <= row < qlen and 0 <= row - k < rlen.
template <int U, bool SMEM>
__device__ __forceinline__ void ext_u(const SeqWin &qs, int32_t qlen, const SeqWin &rs,
                                      int32_t rlen, int32_t (&rows)[U], const int32_t (&ks)[U],
                                      const bool (&live)[U])
{
    // Either sequence empty: no diagonal can extend (and there is no window to load).
    if (qlen <= 0 || rlen <= 0)
        return;
    // Live rows are >= 0 (and so are their columns); dead rows are negative and
    // must not move.  Window positions are clamped into the sequences, so every
    // load is in bounds, and the advance max(0, min(ml, qlen - row, rlen - col))
    // is zeroed for dead rows and for diagonals past the last one.
    int32_t adv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t row = rows[u], col = row - ks[u];
        const int32_t pq = (int32_t)min((uint32_t)row, (uint32_t)(qlen - 1));
        const int32_t pr = (int32_t)min((uint32_t)col, (uint32_t)(rlen - 1));
        const uint32_t x = win16<SMEM>(qs, pq) ^ win16<SMEM>(rs, pr);
        int32_t ml = __clz((int)x) >> 1;
        ml += ml >> 4;  // 17 for a whole matching window
        int32_t a = __vimin3_s32_relu(ml, qlen - row, rlen - col);
        a &= ~(row >> 31);
        if (!live[u])
            a = 0;
        adv[u] = a;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        // 17: the window matched and both sequences go on past it: the rest one by one
        if (adv[u] == 17)
            rows[u] = ext_run<SMEM>(qs, qlen, rs, rlen, rows[u] + 16, ks[u]);
        else
            rows[u] += adv[u];
    }
}

// ---- dump records ---------------------------------------------------------------
// A suspended pair: int32 header {next step, M slot, I/D slot, span lo, span
// hi} at 0, lane j's {M slot j lo, hi, I/D slot j lo, hi} at int 32 + 4j, and
// from byte kDumpHeader the nslot ring rows over [span lo, span hi], each
// span elements of int16.
//
// The shared-memory tiers write the rows with one bulk asynchronous copy per
// row (cp.async.bulk from this CTA's shared memory to global), which needs both
// addresses and the size in whole 16-byte units.  So the span is the live
// span widened outward to diagonals whose window positions H + k are
// multiples of 8: the window's rows start on 16 bytes (W is a multiple of 8,
// the ring 16-byte aligned) and hold positions [0, W), so the widened span
// stays inside the row; outside every slot's interval a row holds NEG, so the
// extra elements are NEG.  Records lie whole multiples of 256 bytes apart and
// the rows at kDumpHeader + j * span * 2 with span a multiple of 8; the
// alignment is checked when a record is written (an element copy otherwise).
// The larger window a record is restored into holds the widened span too (its
// H and W - H are no smaller), where the extra NEGs land on NEG.
__device__ __forceinline__ void bulk_row_to_global(void *dst, const void *src_smem,
                                                   uint32_t bytes)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(src_smem);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 :: "l"(dst), "r"(s), "r"(bytes) : "memory");
}
struct DumpOut {
    uint8_t *base;      // records of dump_stride bytes
    int64_t stride;
    int64_t cap;        // records available
    int *ctr;           // records claimed
};

// ---- one pair ------------------------------------------------------------------
// Aligns pair pi with this team.  ring: the team's window (nslot rows of W
// elements, diagonal k of slot j at ring[j * W + H + k]).  resume: a dump
// record to continue from, or nullptr.  Returns the cost (>= 0), -1 past
// max_error, kPromote (state written to record *dump_idx, or *dump_idx = -1
// when no record was free), or kRestart (int16 rows would overflow).  The
// return value is uniform over the team.
template <int TEAM, int NTEAMS, int U, bool SMEM_SEQ, typename RT>
__device__ __forceinline__ int32_t tier_pair(const SeqView &q, const SeqView &r, const WfaParams &p,
                                             const Shape &w, int64_t pi, RT *ring, int32_t W,
                                             int32_t H, uint2 *sq, uint2 *sr,
                                             const Team<TEAM, NTEAMS> &team,
                                             volatile int64_t *bcast, const uint8_t *resume,
                                             const DumpOut &dump, int64_t *dump_idx,
                                             int64_t &cells, int32_t band_w, int32_t ub)
{
    constexpr int TW = TEAM * 32;
    constexpr int32_t NEG = Neg<RT>::value;
    constexpr bool R16 = std::is_same<RT, int16_t>::value;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tt = (int)(threadIdx.x % TW);
    const int hm = w.hm, hie = w.hie, xs = w.xs, oes = w.oes, es = w.es, g = w.g;
    const int32_t max_err = p.max_error;
    const int64_t qoff = q.offsets[pi] - q.word_base;
    const int64_t roff = r.offsets[pi] - r.word_base;
    const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
    if (qlen == 0 && rlen == 0)
        return 0;
    const int32_t qnw = (qlen + 31) >> 5, rnw = (rlen + 31) >> 5;
    team.sync();  // the previous pair's reads of the shared copies and the ring are done
    const SeqWin qs = stage_seq<SMEM_SEQ>(q, qoff, qnw, sq, tt, TW);
    const SeqWin rs = stage_seq<SMEM_SEQ>(r, roff, rnw, sr, tt, TW);
    // every ring element NEG
    {
        const int32_t total = (w.nslot + 1) * W;  // the slots and the NEG row
        if (R16) {
            // W is a multiple of 8 and the window 16-byte aligned
            uint4 *v = reinterpret_cast<uint4 *>(ring);
            const uint4 n4 = make_uint4(0x80008000u, 0x80008000u, 0x80008000u, 0x80008000u);
            for (int32_t i = tt; i < total / 8; i += TW)
                v[i] = n4;
        } else {
            for (int32_t i = tt; i < total; i += TW)
                ring[i] = (RT)NEG;
        }
    }
    const int32_t target = qlen - rlen;
    RT *const base = ring + H;
    auto slot = [&](int j) { return base + j * W; };
    // per-slot intervals: lane j holds M slot j's and I/D slot j's
    int32_t mlo = 1, mhi = 0, ilo = 1, ihi = 0;
    int ms = 0, is = 0;
    int64_t sp0 = 1;
    int32_t result = kRunning;
    team.sync();  // NEG fill done before the restored / initial values land
    if (resume) {
        const int32_t *hd = reinterpret_cast<const int32_t *>(resume);
        sp0 = hd[0];
        ms = hd[1];
        is = hd[2];
        const int32_t ulo = hd[3], uhi = hd[4];
        mlo = hd[32 + 4 * lane];
        mhi = hd[33 + 4 * lane];
        ilo = hd[34 + 4 * lane];
        ihi = hd[35 + 4 * lane];
        const int32_t span = uhi - ulo + 1;
        if (span > 0) {
            const RT *src = reinterpret_cast<const RT *>(resume + kDumpHeader);
            const int32_t total = w.nslot * span;
            for (int32_t i = tt; i < total; i += TW) {
                const int32_t j = i / span, kk = i - j * span;
                slot(j)[ulo + kk] = src[i];
            }
        }
    } else {
        // score 0: M[0,0] = 0 extended along diagonal 0 (:130-140)
        const int32_t row0 = ext_run<SMEM_SEQ>(qs, qlen, rs, rlen, 0, 0);
        if (lane == 0) {
            mlo = 0;
            mhi = 0;
        }
        if (tt == 0)
            slot(0)[0] = (RT)row0;
        cells += 1;
        if (target == 0 && row0 >= qlen)
            result = 0;
    }
    team.sync();
    int32_t rq = 0, rr = 0;  // pruning: (ub - s) / e and its remainder at s = sp0 * g
    if (ub >= 0) {
        const int32_t num = ub - (int32_t)(sp0 * g);
        rq = num / p.e;
        rr = num - rq * p.e;
    }
    if (result == kRunning) {
        // steps s = sp * g <= max_err; int16 rows are proven for sp <= 32767 - qlen
        const int32_t sp_end = max_err / g;
        const int32_t sp_lim = R16 ? min(sp_end, 32767 - qlen) : sp_end;
        int32_t sp = (int32_t)sp0;
        for (; sp <= sp_lim; ++sp) {
            const int32_t s = (int32_t)(sp * g);
            const int nms = ms + 1 == hm ? 0 : ms + 1;
            const int nis = is + 1 == hie ? 0 : is + 1;
            int32_t lo = max(-rlen, -s), hi = min(qlen, s);
            if (target < lo || target > hi) {
                lo = min(lo, target);
                hi = max(hi, target);
            }
            lo = max(lo, -max_err);
            hi = min(hi, max_err);
            if (band_w > 0) {
                // the bound pass: only the band around the line from diagonal 0 to
                // the target, which still holds real alignments (their costs bound
                // the optimum from above)
                lo = max(lo, min(0, target) - band_w);
                hi = min(hi, max(0, target) + band_w);
            }
            if (ub >= 0) {
                // a diagonal k at score s costs at least s + e*|k - target| to finish
                // (every diagonal change is a gap base): beyond the upper bound ub it
                // cannot be on an alignment of cost <= ub, and dropping it only
                // lowers values elsewhere, so the first hit stays at the same s
                // R = (ub - s) / e, kept as quotient and remainder (s grows by g
                // per step, and ub >= s while the pair runs)
                const int32_t R = rq;
                rr -= g;
                if (rr < 0) {
                    rr += p.e;
                    --rq;
                }
                lo = max(lo, target - R);
                hi = min(hi, target + R);
            }
            const int sx = sp >= xs ? (nms >= xs ? nms - xs : nms - xs + hm) : -1;
            const int soe = sp >= oes ? (nms >= oes ? nms - oes : nms - oes + hm) : -1;
            const int se = sp >= es ? (nis >= es ? nis - es : nis - es + hie) : -1;
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
            // this step reads [a-1, b+1] and writes [a, b]: outside the window
            // the pair moves to the next tier, in the state after step sp-1
            if (a <= b && (a - 1 < -H || b + 1 > W - 1 - H)) {
                int64_t di = -1;
                if (dump.base) {
                    if (tt == 0) {
                        const int64_t c = atomicAdd(dump.ctr, 1);
                        *bcast = c < dump.cap ? c : -1;
                    }
                    team.sync();
                    di = *bcast;
                    team.sync();  // read by every thread before the slot is reused
                }
                if (di >= 0) {
                    uint8_t *rec = dump.base + di * dump.stride;
                    int32_t *hd = reinterpret_cast<int32_t *>(rec);
                    // the live span: the union of every slot's interval
                    int32_t l0 = 0x7fffffff, h0 = -0x7fffffff;
                    if (lane < hm && mlo <= mhi) {
                        l0 = mlo;
                        h0 = mhi;
                    }
                    if (lane < hie && ilo <= ihi) {
                        l0 = min(l0, ilo);
                        h0 = max(h0, ihi);
                    }
                    l0 = __reduce_min_sync(FULL, l0);
                    h0 = __reduce_max_sync(FULL, h0);
                    if (R16 && l0 <= h0) {  // widen to 16-byte units of the window rows
                        l0 -= (H + l0) & 7;
                        h0 += 7 - ((H + h0) & 7);
                    }
                    if (tt == 0) {
                        hd[0] = (int32_t)sp;
                        hd[1] = ms;
                        hd[2] = is;
                        hd[3] = l0;
                        hd[4] = h0;
                    }
                    if (tt < 32) {
                        hd[32 + 4 * lane] = mlo;
                        hd[33 + 4 * lane] = mhi;
                        hd[34 + 4 * lane] = ilo;
                        hd[35 + 4 * lane] = ihi;
                    }
                    const int32_t span = h0 - l0 + 1;
                    if (span > 0) {
                        int16_t *dst = reinterpret_cast<int16_t *>(rec + kDumpHeader);
                        // alignment as derived above, checked (the same on every thread
                        // of the team): the element copy below otherwise
                        const bool bulk =
                            R16 && (((uintptr_t)dst & 15u) == 0) && ((W & 7) == 0) &&
                            ((__cvta_generic_to_shared(slot(0) + l0) & 15u) == 0);
                        if (bulk) {
                            // every thread orders its ring writes before the async
                            // proxy's reads, then one thread hands the rows to the
                            // copy engine and waits for them before the team can
                            // reuse the window (the next pair starts with a barrier)
                            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                            team.sync();
                            if (tt == 0) {
                                for (int j = 0; j < w.nslot; ++j)
                                    bulk_row_to_global(dst + (int64_t)j * span, slot(j) + l0,
                                                       (uint32_t)span * 2u);
                                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                                asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
                            }
                        } else {
                            const int32_t total = w.nslot * span;
                            for (int32_t i = tt; i < total; i += TW) {
                                const int32_t j = i / span, kk = i - j * span;
                                dst[i] = (int16_t)slot(j)[l0 + kk];
                            }
                        }
                    }
                }
                *dump_idx = di;
                result = kPromote;
                break;
            }
            ms = nms;
            is = nis;
            const int32_t omlo = __shfl_sync(FULL, mlo, ms);
            const int32_t omhi = __shfl_sync(FULL, mhi, ms);
            const int32_t oilo = __shfl_sync(FULL, ilo, is);
            const int32_t oihi = __shfl_sync(FULL, ihi, is);
            RT *const Mw = slot(ms);
            RT *const Iw = slot(hm + is);
            RT *const Dw = slot(hm + hie + is);
            // what the reused slots held outside [a, b] becomes NEG (all of it
            // when this score is empty)
            const int32_t ca = a > b ? 0x7fffffff : a, cb = a > b ? -0x7fffffff : b;
            if ((omlo <= omhi && (omlo < ca || omhi > cb)) ||
                (oilo <= oihi && (oilo < ca || oihi > cb))) {
                for (int32_t k = omlo + tt; k <= min(omhi, ca - 1); k += TW)
                    Mw[k] = (RT)NEG;
                for (int32_t k = max(omlo, cb + 1) + tt; k <= omhi; k += TW)
                    Mw[k] = (RT)NEG;
                for (int32_t k = oilo + tt; k <= min(oihi, ca - 1); k += TW) {
                    Iw[k] = (RT)NEG;
                    Dw[k] = (RT)NEG;
                }
                for (int32_t k = max(oilo, cb + 1) + tt; k <= oihi; k += TW) {
                    Iw[k] = (RT)NEG;
                    Dw[k] = (RT)NEG;
                }
            }
            bool hit = false;
            if (a <= b) {
                cells += (int64_t)(b - a + 1);
                // a source that does not exist yet reads the row kept NEG (slot nslot)
                const RT *negrow = slot(w.nslot);
                const RT *Mx = sx >= 0 ? slot(sx) : negrow;
                const RT *Moe = soe >= 0 ? slot(soe) : negrow;
                const RT *Ie = se >= 0 ? slot(hm + se) : negrow;
                const RT *De = se >= 0 ? slot(hm + hie + se) : negrow;
                // rounds of UU diagonals per thread: full rounds (every diagonal
                // inside [a, b]) while they last, then single-diagonal rounds
                auto round = [&](int32_t k0, auto uc, auto fc) {
                    constexpr int UU = decltype(uc)::value;
                    constexpr bool FULLR = decltype(fc)::value;
                    int32_t ks[UU], iv[UU], dv[UU], mv[UU];
                    bool live[UU];
#pragma unroll
                    for (int u = 0; u < UU; ++u) {
                        ks[u] = k0 + TW * u;
                        live[u] = FULLR || ks[u] <= b;
                        const int32_t kc = FULLR ? ks[u] : (live[u] ? ks[u] : b);
                        const int32_t io = (int32_t)Moe[kc - 1], dop = (int32_t)Moe[kc + 1];
                        const int32_t ie = (int32_t)Ie[kc - 1], dex = (int32_t)De[kc + 1];
                        const int32_t mx = (int32_t)Mx[kc];
                        const int32_t i0 = max(io, ie), d0 = max(dop, dex);
                        // max(mx + 1, i0 + 1, d0) as two DPX add-max instructions
                        const int32_t m1 = __viaddmax_s32(mx, 1, __viaddmax_s32(i0, 1, d0));
                        if (R16) {
                            iv[u] = i0 + 1;
                            mv[u] = m1;
                        } else {
                            iv[u] = i0 < 0 ? NEG : i0 + 1;
                            mv[u] = m1 < 0 ? NEG : m1;
                        }
                        dv[u] = d0;
                    }
                    ext_u<UU, SMEM_SEQ>(qs, qlen, rs, rlen, mv, ks, live);
#pragma unroll
                    for (int u = 0; u < UU; ++u) {
                        if (live[u]) {
                            Iw[ks[u]] = (RT)iv[u];
                            Dw[ks[u]] = (RT)dv[u];
                            Mw[ks[u]] = (RT)mv[u];
                        }
                    }
                };
                int32_t k0 = a + tt;
                for (; k0 + TW * (U - 1) <= b; k0 += TW * U)
                    round(k0, std::integral_constant<int, U>{}, std::true_type{});
                for (; k0 <= b; k0 += TW)
                    round(k0, std::integral_constant<int, 1>{}, std::false_type{});
                // the thread that owns the target diagonal reads back its own store
                if ((uint32_t)(target - a) <= (uint32_t)(b - a) && ((target - a) & (TW - 1)) == tt)
                    hit = (int32_t)Mw[target] >= qlen;
            }
            if (lane == ms) {
                mlo = a <= b ? a : 1;
                mhi = a <= b ? b : 0;
            }
            if (lane == is) {
                ilo = a <= b ? a : 1;
                ihi = a <= b ? b : 0;
            }
            // M[s, target] >= qlen ends the alignment (:221-224)
            if (team.any(hit)) {
                result = s;
                break;
            }
        }
        if (result == kRunning)
            result = sp <= sp_end ? kRestart  // past the steps int16 values are proven for
                                  : -1;       // the loop ran out: cost above max_error (:226)
    }
    return result;
}

// ---- tier kernel -----------------------------------------------------------------
// Work items: the pairs of `list` (int32 pair indices; nullptr = 0..n-1) or of
// `ents` ({pair, dump record or -1}); n from the host, or from *n_dev when
// set.  Items are handed out by atomics on ctr.
struct TierIn {
    const int32_t *list;
    const int2 *ents;
    int64_t n;
    const int *n_dev;
    const int64_t *seg;     // when set: list + seg[0], n = seg[1] - seg[0]
    int *ctr;
    const uint8_t *dumps;   // records the entries refer to
    int64_t dump_stride;
    const int32_t *ubound;  // per pair: a cost no lower than the optimum (-1: max_error)
    int32_t band_w;         // > 0: the bound pass's band half-width
};

struct TierOut {
    int2 *next;      // queue of the next tier
    int *next_n;
    DumpOut dump;    // records of pairs suspended here (base nullptr: none)
    int2 *restart;   // the G tier's queue
    int *restart_n;
};

struct TierGeom {
    int32_t W, H;           // window: elements per slot row, offset of diagonal 0
    int64_t team_bytes;     // shared bytes of one team (ring + sequence copies)
    int64_t ring_bytes;     // of them, the ring (shared) -- 0 for the G tier
    int32_t seq_cap;        // 16-base window entries per sequence copy
    int32_t *gring;         // G tier: per-block int32 regions of nslot * W
};

template <int TEAM, int NTEAMS, typename RT, bool GRING>
__global__ void __launch_bounds__(TEAM *NTEAMS * 32, 1)
wfa_tier_kernel(SeqView q, SeqView r, WfaParams p, TierIn in, TierOut tout, TierGeom geo,
                int32_t *__restrict__ out, int64_t *work, int *err_flag)
{
    extern __shared__ __align__(16) uint8_t tsm[];
    __shared__ int64_t bcast[NTEAMS];
    const Shape w = make_shape(p);
    const int team_id = (int)(threadIdx.x / (TEAM * 32));
    const int tt = (int)(threadIdx.x % (TEAM * 32));
    const Team<TEAM, NTEAMS> team{team_id};
    uint8_t *const mine = tsm + team_id * geo.team_bytes;
    RT *ring;
    if (GRING)
        ring = reinterpret_cast<RT *>(geo.gring +
                                      (int64_t)blockIdx.x * (w.nslot + 1) * (int64_t)geo.W);
    else
        ring = reinterpret_cast<RT *>(mine);
    uint2 *const sq = reinterpret_cast<uint2 *>(mine + geo.ring_bytes);
    uint2 *const sr = sq + geo.seq_cap;
    int64_t n = in.n;
    const int32_t *list = in.list;
    if (in.seg) {
        list = in.list + in.seg[0];
        n = in.seg[1] - in.seg[0];
    }
    if (in.n_dev)
        n = *in.n_dev;
    int64_t cells = 0;
    volatile int64_t *bc = &bcast[team_id];
    for (;;) {
        if (tt == 0)
            *bc = atomicAdd(in.ctr, 1);
        team.sync();
        const int64_t it = *bc;
        team.sync();  // every thread has read the slot before it is reused
        if (it >= n)
            break;
        int64_t pi;
        const uint8_t *resume = nullptr;
        if (in.ents) {
            const int2 e = in.ents[it];
            pi = e.x;
            if (e.y >= 0 && in.dumps)
                resume = in.dumps + (int64_t)e.y * in.dump_stride;
        } else {
            pi = list ? (int64_t)list[it] : it;
        }
        const int64_t ql = q.lengths[pi], rl = r.lengths[pi];
        const bool smem_seq = 2 * ((ql + 31) >> 5) <= geo.seq_cap &&
                              2 * ((rl + 31) >> 5) <= geo.seq_cap;
        int64_t di = -2;
        int32_t res;
        int32_t ub = -1;
        if (in.ubound) {
            ub = in.ubound[pi];
            if (ub < 0)
                ub = p.max_error;
        }
        if (smem_seq)
            res = tier_pair<TEAM, NTEAMS, 4, true, RT>(q, r, p, w, pi, ring, geo.W, geo.H, sq, sr,
                                                       team, bc, resume, tout.dump, &di, cells,
                                                       in.band_w, ub);
        else
            res = tier_pair<TEAM, NTEAMS, 4, false, RT>(q, r, p, w, pi, ring, geo.W, geo.H, sq, sr,
                                                        team, bc, resume, tout.dump, &di, cells,
                                                        in.band_w, ub);
        if (tt == 0) {
            if (res >= -1) {
                out[pi] = res;
            } else if (res == kPromote && tout.next) {
                const int slot = atomicAdd(tout.next_n, 1);
                tout.next[slot] = make_int2((int)pi, (int)di);
            } else if (tout.restart) {
                // kRestart, or a window overflow with no tier above: the G tier
                const int slot = atomicAdd(tout.restart_n, 1);
                tout.restart[slot] = make_int2((int)pi, -1);
            } else if (in.band_w > 0) {
                out[pi] = -1;  // the bound pass could not finish this pair: no bound
            } else {
                out[pi] = -3;  // no tier left (the G window holds every diagonal)
                atomicOr(err_flag, 1);
            }
        }
    }
    if (tt == 0 && work && cells)
        atomicAdd((unsigned long long *)work, (unsigned long long)cells);
}

}  // namespace

// ---- host side --------------------------------------------------------------------
// Shared memory of one block (the device maximum per block, less a margin for
// the kernel's static shared variables).
constexpr int64_t kTierBlockSmem = 227 * 1024 - 256;

struct TierSpec {
    int team_warps, nteams;
    int32_t seq_bases;  // longest sequence copied to shared memory
};
// S, M, L tiers
static const TierSpec kTiers[kWfaShared] = {{1, 16, 2048}, {2, 8, 4096}, {4, 4, 8192}, {8, 2, 16384}, {16, 1, 32768}};

WfaTierPlan wfa_tier_plan(const WfaParams &p, int64_t qmax, int64_t rmax)
{
    auto gcd_h = [](int a, int b) {
        while (b) {
            const int t = a % b;
            a = b;
            b = t;
        }
        return a;
    };
    const int g = gcd_h(p.x, gcd_h(p.o, p.e));
    const int hm = std::max(p.x / g, (p.o + p.e) / g) + 1, hie = p.e / g + 1;
    const int nslot = hm + 2 * hie;
    WfaTierPlan plan{};
    plan.nslot = nslot;
    for (int t = 0; t < kWfaShared; ++t) {
        const TierSpec &s = kTiers[t];
        const int64_t team_bytes = kTierBlockSmem / s.nteams;
        const int64_t seq_entries = 2 * ((s.seq_bases + 31) / 32);  // halves per sequence
        const int64_t seq_bytes = 2 * seq_entries * 8;
        int64_t W = (team_bytes - seq_bytes) / ((nslot + 1) * 2);
        W = W / 8 * 8;  // 16-byte rows: the NEG fill uses 16-byte stores
        plan.W[t] = (int32_t)W;
        plan.H[t] = (int32_t)(W / 2 - 1);
        plan.seq_cap[t] = (int32_t)seq_entries;
        plan.team_bytes[t] = team_bytes & ~int64_t(15);
        plan.ring_bytes[t] = (int64_t)(nslot + 1) * W * 2;
        plan.usable[t] = W >= 64;
        plan.dump_stride[t] = (kDumpHeader + (int64_t)nslot * W * 2 + 255) & ~int64_t(255);
    }
    // G: int32 rings covering [-max(qlen, rlen) - 3, max(qlen, rlen) + 3]
    const int64_t lmax = std::max(qmax, rmax);
    constexpr int G = kWfaShared;
    plan.W[G] = (int32_t)(((2 * lmax + 8) + 7) & ~int64_t(7));
    plan.H[G] = (int32_t)(lmax + 3);
    plan.seq_cap[G] = (int32_t)(2 * ((kTiers[G - 1].seq_bases + 31) / 32));
    plan.team_bytes[G] = 2 * (int64_t)plan.seq_cap[G] * 8;
    plan.ring_bytes[G] = 0;
    plan.usable[G] = true;
    plan.gring_block_bytes = (int64_t)(nslot + 1) * plan.W[G] * 4;
    return plan;
}

template <int TEAM, int NTEAMS, typename RT, bool GRING>
static cudaError_t tier_launch(const WfaTierPlan &pl, int t, int grid, SeqView q, SeqView r,
                               WfaParams p, const TierIn &in, const TierOut &o, int32_t *gring,
                               int32_t *out, int64_t *work, int *err_flag, cudaStream_t st)
{
    const size_t smem = (size_t)pl.team_bytes[t] * NTEAMS;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(wfa_tier_kernel<TEAM, NTEAMS, RT, GRING>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTierBlockSmem);
        attr = true;
    }
    TierGeom geo{pl.W[t], pl.H[t], pl.team_bytes[t], pl.ring_bytes[t], pl.seq_cap[t], gring};
    wfa_tier_kernel<TEAM, NTEAMS, RT, GRING><<<grid, TEAM * NTEAMS * 32, smem, st>>>(
        q, r, p, in, o, geo, out, work, err_flag);
    return cudaGetLastError();
}

cudaError_t launch_wfa_tier(const WfaTierPlan &pl, int tier, int grid, SeqView q, SeqView r,
                            WfaParams p, const WfaTierIo &io, int32_t *out, int64_t *work,
                            int *err_flag, cudaStream_t st)
{
    TierIn in{io.list,    io.ents,           io.n,      io.n_dev, io.seg,
              io.ctr,     io.dumps_in,       io.dump_in_stride,   io.ubound, io.band_w};
    TierOut o{io.next, io.next_n, DumpOut{io.dumps_out, io.dump_out_stride, io.dump_out_cap,
                                          io.dump_out_ctr},
              io.restart, io.restart_n};
    switch (tier) {
    case 0:
        return tier_launch<1, 16, int16_t, false>(pl, 0, grid, q, r, p, in, o, nullptr, out,
                                                  work, err_flag, st);
    case 1:
        return tier_launch<2, 8, int16_t, false>(pl, 1, grid, q, r, p, in, o, nullptr, out,
                                                 work, err_flag, st);
    case 2:
        return tier_launch<4, 4, int16_t, false>(pl, 2, grid, q, r, p, in, o, nullptr, out,
                                                 work, err_flag, st);
    case 3:
        return tier_launch<8, 2, int16_t, false>(pl, 3, grid, q, r, p, in, o, nullptr, out,
                                                 work, err_flag, st);
    case 4:
        return tier_launch<16, 1, int16_t, false>(pl, 4, grid, q, r, p, in, o, nullptr, out,
                                                  work, err_flag, st);
    default:
        return tier_launch<16, 1, int32_t, true>(pl, kWfaShared, grid, q, r, p, in, o, io.gring,
                                                 out, work, err_flag, st);
    }
}

}  // namespace gb2
