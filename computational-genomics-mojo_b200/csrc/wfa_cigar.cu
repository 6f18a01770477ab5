// wfa_cigar.cu -- gap-affine WFA with CIGAR traceback on sm_100a.
//
// wfa_affine_cigar_cpu (genomics/cpu/align_cpu.mojo:380-623) keeps M before
// and after extension, I and D for every score up to the optimum and every
// diagonal in [-max_err, max_err], then walks back from (opt, qlen - rlen).
// Here a first pass is the cost kernel, which also reports how many bytes
// each pair's history will take; a second pass re-runs the forward
// recurrences (same visited intervals and rings as the cost kernel, one warp
// per pair) and appends, for every visited score, the M-after-extension
// values and one decision byte per diagonal to the pair's history record in
// an arena sized from the first pass.  The decision byte records what the
// reference's traceback finds by comparing values (:509-601):
//   * M before extension came from the mismatch source when M[s-x, k] + 1
//     equals it, else from I when I[s, k] equals it, else from D;
//   * I[s, k] came from an open when M[s-o-e, k-1] + 1 equals it, else from
//     an extension I[s-e, k-1] + 1;
//   * D[s, k] came from an open when M[s-o-e, k+1] equals it, else from
//     D[s-e, k+1]
// (the same priority order as the traceback's tests).  With those bytes the
// traceback needs only M-after values:
//   M state (s, k), current row = M-after[s, k]: the row before extension is
//     (mismatch) M-after[s-x, k] + 1; (I) follow the I chain back to its
//     open (s', k'): M-after[s'-o-e, k'-1] + 1 + number of extensions;
//     (D) the D chain's open: M-after[s'-o-e, k'+1].  Emit (row - before)
//     '=' ops, then 'X' and go to (s-x, k), or enter I or D;
//   I state: one 'I', then M at (s-o-e, k-1) or I at (s-e, k-1);
//   D state: one 'D', then M at (s-o-e, k+1) or D at (s-e, k+1);
// ending at score 0, diagonal 0.  Ops come out back to front and are
// run-length encoded as the reference does (:603-621): a run is
// len << 2 | op, op 0 '=', 1 'X', 2 'I', 3 'D'.
//
// A history record costs 4 B + 1 B per visited cell plus 12 B per score,
// against the reference's 4 int64 arrays over (max_err+1) x (2 max_err+1).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "runtime.cuh"

namespace gb2 {

#define WFA_NEG_C (-(1 << 30))

namespace {

__device__ __forceinline__ int gcd_c(int a, int b)
{
    while (b) {
        int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

struct Halves {
    const uint32_t *w;
    int32_t last;
    uint32_t swz;
};

// 16 bases at pos (see the cost kernel's window16: halves high first in
// shared memory, swz = 1 for the little-endian words in global memory).
__device__ __forceinline__ uint32_t win16(const Halves &s, int32_t pos)
{
    const int32_t j = pos >> 4;
    const uint32_t hi = s.w[(uint32_t)j ^ s.swz];
    const uint32_t lo = s.w[(uint32_t)min(j + 1, s.last) ^ s.swz];
    return __funnelshift_l(lo, hi, (uint32_t)(pos & 15) << 1);
}

// Extend along diagonal k from row (align_cpu.mojo:489-498).
__device__ __forceinline__ int32_t extend16(const Halves &qs, int32_t qlen, const Halves &rs,
                                            int32_t rlen, int32_t row, int32_t k)
{
    if (row < 0 || row - k < 0)
        return row;
    int32_t col = row - k;
    while (row < qlen && col < rlen) {
        const uint32_t x = win16(qs, row) ^ win16(rs, col);
        const int ml = x ? (__clz((int)x) >> 1) : 16;
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

constexpr int kSeqWords = 321;  // per sequence per warp: 10,240 bases + a zero pad

__device__ __forceinline__ Halves stage(const SeqView &v, int64_t off, int32_t nw, uint32_t *smem,
                                        int lane)
{
    if (nw < kSeqWords) {
        uint2 *d = reinterpret_cast<uint2 *>(smem);
        for (int i = lane; i <= nw; i += 32) {
            const uint64_t x = i < nw ? __ldg(v.packed + off + i) : 0;
            d[i] = make_uint2((uint32_t)(x >> 32), (uint32_t)x);
        }
        return Halves{smem, 2 * nw, 0u};
    }
    const int64_t last = 2 * (v.n_words - off) - 1;
    return Halves{reinterpret_cast<const uint32_t *>(v.packed + off),
                  (int32_t)min(last, (int64_t)0x7fffffff), 1u};
}

// Read access to one pair's history record.
struct Hist {
    const uint8_t *rec;
    const int32_t *hdr;
    __device__ __forceinline__ int32_t mafter(int sp, int32_t k) const
    {
        if (sp < 0)
            return WFA_NEG_C;
        const int32_t a = hdr[3 * sp], b = hdr[3 * sp + 1];
        if (k < a || k > b)
            return WFA_NEG_C;
        return reinterpret_cast<const int32_t *>(rec)[hdr[3 * sp + 2] + (k - a)];
    }
    __device__ __forceinline__ uint32_t dec(int sp, int32_t k) const
    {
        if (sp < 0)
            return 0;
        const int32_t a = hdr[3 * sp], b = hdr[3 * sp + 1];
        if (k < a || k > b)
            return 0;
        const int64_t off = hdr[3 * sp + 2];
        return rec[(off + (b - a + 1)) * 4 + (k - a)];
    }
};

__global__ void __launch_bounds__(128)
wfa_cigar_kernel(SeqView q, SeqView r, WfaParams p, const int32_t *__restrict__ pairs, int64_t n,
                 int *counter, const int32_t *__restrict__ cost,
                 const int64_t *__restrict__ hist_cells, const int64_t *__restrict__ arena_off,
                 uint8_t *__restrict__ arena, int32_t *__restrict__ scratch, int64_t slot_width,
                 uint32_t *__restrict__ runs, const int64_t *__restrict__ run_off,
                 int32_t *__restrict__ run_count, int *err_flag)
{
    __shared__ __align__(16) uint32_t seqs[4 * 2 * 2 * kSeqWords];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int g = gcd_c(p.x, gcd_c(p.o, p.e));
    const int xs = p.x / g, oes = (p.o + p.e) / g, es = p.e / g;
    const int hm = max(xs, oes) + 1, hie = es + 1;
    const int nslot = hm + 2 * hie;
    int32_t *const region = scratch + ((int64_t)blockIdx.x * 4 + wib) * nslot * slot_width;
    uint32_t *const my = seqs + wib * 4 * kSeqWords;

    for (;;) {
        int64_t b0 = 0;
        if (lane == 0)
            b0 = atomicAdd(counter, 1);
        const int64_t si = __shfl_sync(FULL, b0, 0);
        if (si >= n)
            break;
        const int64_t pi = pairs[si];
        const int32_t c = cost[pi];
        const int64_t qoff = q.offsets[pi] - q.word_base;
        const int64_t roff = r.offsets[pi] - r.word_base;
        const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
        if (c < 0 || (qlen == 0 && rlen == 0)) {
            if (lane == 0)
                run_count[pi] = 0;
            continue;
        }
        if ((int64_t)qlen + rlen + 5 > slot_width || c % g != 0) {
            if (lane == 0) {
                atomicOr(err_flag, 1);
                run_count[pi] = -1;
            }
            continue;
        }
        const int S = c / g + 1;  // visited score indices 0 .. c/g
        uint8_t *const rec = arena + arena_off[pi];
        int32_t *const hdr = reinterpret_cast<int32_t *>(rec);
        int32_t *const recw = reinterpret_cast<int32_t *>(rec);
        int64_t cur = 3 * (int64_t)S;  // next free 4-byte word of the record
        // the record's size from the cost pass; a step that would pass it
        // (the two passes disagree) stops the pair with an error instead
        const int64_t limit = cur + hist_cells[pi] / 4;
        bool overrun = false;

        __syncwarp();  // the previous pair's reads of the shared copies are done
        const Halves qs = stage(q, qoff, (qlen + 31) >> 5, my, lane);
        const Halves rs = stage(r, roff, (rlen + 31) >> 5, my + 2 * kSeqWords, lane);
        const int32_t kofs = rlen + 2;
        const int32_t target = qlen - rlen;
        int32_t *const base = region + kofs;
        auto M = [&](int slot) { return base + (int64_t)slot * slot_width; };
        auto I = [&](int slot) { return base + (int64_t)(hm + slot) * slot_width; };
        auto D = [&](int slot) { return base + (int64_t)(hm + hie + slot) * slot_width; };
        int32_t mlo = 1, mhi = 0, ilo = 1, ihi = 0;
        int32_t GL = max(-2, -rlen - 2), GH = min(2, qlen + 2);
        for (int sl = 0; sl < nslot; ++sl) {
            int32_t *row = base + (int64_t)sl * slot_width;
            for (int32_t k = GL + lane; k <= GH; k += 32)
                row[k] = WFA_NEG_C;
        }
        __syncwarp();
        const int32_t row0 = extend16(qs, qlen, rs, rlen, 0, 0);
        if (lane == 0) {  // score 0 (cur + 2 <= limit: the cost pass counts 8 bytes for it)
            mlo = 0;
            mhi = 0;
            M(0)[0] = row0;
            hdr[0] = 0;
            hdr[1] = 0;
            hdr[2] = (int32_t)cur;
            recw[cur] = row0;
            rec[(cur + 1) * 4] = 0;
        }
        cur += wfa_hist_cell_bytes(1) / 4;
        __syncwarp();
        int32_t result = (target == 0 && row0 >= qlen) ? 0 : -1;
        int ms = 0, is = 0;
        for (int sp = 1; result < 0 && sp < S; ++sp) {
            const int32_t s = sp * g;
            ms = ms + 1 == hm ? 0 : ms + 1;
            is = is + 1 == hie ? 0 : is + 1;
            int32_t lo = max(-rlen, -s), hi = min(qlen, s);
            if (target < lo || target > hi) {
                lo = min(lo, target);
                hi = max(hi, target);
            }
            lo = max(lo, -p.max_error);
            hi = min(hi, p.max_error);
            const int sx = sp >= xs ? (ms >= xs ? ms - xs : ms - xs + hm) : -1;
            const int soe = sp >= oes ? (ms >= oes ? ms - oes : ms - oes + hm) : -1;
            const int se = sp >= es ? (is >= es ? is - es : is - es + hie) : -1;
            int32_t ulo = 0x7fffffff, uhi = -0x7fffffff;
            {
                const int32_t a0 = __shfl_sync(FULL, mlo, sx & 31);
                const int32_t b0v = __shfl_sync(FULL, mhi, sx & 31);
                if (sx >= 0 && a0 <= b0v) {
                    ulo = a0;
                    uhi = b0v;
                }
                const int32_t a1 = __shfl_sync(FULL, mlo, soe & 31);
                const int32_t b1 = __shfl_sync(FULL, mhi, soe & 31);
                if (soe >= 0 && a1 <= b1) {
                    ulo = min(ulo, a1 - 1);
                    uhi = max(uhi, b1 + 1);
                }
                const int32_t a2 = __shfl_sync(FULL, ilo, se & 31);
                const int32_t b2 = __shfl_sync(FULL, ihi, se & 31);
                if (se >= 0 && a2 <= b2) {
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
            int32_t *const Mw = M(ms), *const Iw = I(is), *const Dw = D(is);
            const int32_t ca = a > b ? 0x7fffffff : a, cb = a > b ? -0x7fffffff : b;
            for (int32_t k = omlo + lane; k <= min(omhi, ca - 1); k += 32)
                Mw[k] = WFA_NEG_C;
            for (int32_t k = max(omlo, cb + 1) + lane; k <= omhi; k += 32)
                Mw[k] = WFA_NEG_C;
            for (int32_t k = oilo + lane; k <= min(oihi, ca - 1); k += 32) {
                Iw[k] = WFA_NEG_C;
                Dw[k] = WFA_NEG_C;
            }
            for (int32_t k = max(oilo, cb + 1) + lane; k <= oihi; k += 32) {
                Iw[k] = WFA_NEG_C;
                Dw[k] = WFA_NEG_C;
            }
            if (lane == 0) {
                hdr[3 * sp] = a <= b ? a : 1;
                hdr[3 * sp + 1] = a <= b ? b : 0;
                hdr[3 * sp + 2] = a <= b ? (int32_t)cur : 0;
            }
            bool hit = false;
            if (a <= b && cur + wfa_hist_cell_bytes(b - a + 1) / 4 > limit) {
                overrun = true;  // same decision in every lane
                break;
            }
            if (a <= b) {
                const int32_t wdt = b - a + 1;
                int32_t *const hm_out = recw + cur;
                uint8_t *const hd_out = rec + (cur + wdt) * 4;
                const int32_t *Mx = sx >= 0 ? M(sx) : nullptr;
                const int32_t *Moe = soe >= 0 ? M(soe) : nullptr;
                const int32_t *Ie = se >= 0 ? I(se) : nullptr;
                const int32_t *De = se >= 0 ? D(se) : nullptr;
                for (int32_t k = a + lane; k <= b; k += 32) {
                    int32_t io = WFA_NEG_C, ie = WFA_NEG_C, dop = WFA_NEG_C, dex = WFA_NEG_C,
                            mx = WFA_NEG_C;
                    if (Moe) {
                        io = Moe[k - 1];
                        dop = Moe[k + 1];
                    }
                    if (Ie) {
                        ie = Ie[k - 1];
                        dex = De[k + 1];
                    }
                    if (Mx)
                        mx = Mx[k];
                    const int32_t io1 = io < 0 ? WFA_NEG_C : io + 1;
                    const int32_t ie1 = ie < 0 ? WFA_NEG_C : ie + 1;
                    const int32_t iv = max(io1, ie1);
                    const int32_t dv = max(dop < 0 ? WFA_NEG_C : dop, dex < 0 ? WFA_NEG_C : dex);
                    const int32_t mx1 = mx < 0 ? WFA_NEG_C : mx + 1;
                    const int32_t mpre = max(mx1, max(iv, dv));
                    uint32_t dec = 0;
                    if (mpre >= 0)
                        dec = (mx1 >= 0 && mx1 == mpre) ? 1u : ((iv >= 0 && iv == mpre) ? 2u : 3u);
                    if (iv >= 0 && !(io1 >= 0 && io1 == iv))
                        dec |= 4u;
                    if (dv >= 0 && !(dop >= 0 && dop == dv))
                        dec |= 8u;
                    const int32_t mv =
                        mpre >= 0 ? extend16(qs, qlen, rs, rlen, mpre, k) : WFA_NEG_C;
                    Iw[k] = iv;
                    Dw[k] = dv;
                    Mw[k] = mv;
                    hm_out[k - a] = mv;
                    hd_out[k - a] = (uint8_t)dec;
                    hit |= k == target && mv >= qlen;
                }
                cur += wfa_hist_cell_bytes(wdt) / 4;
                if (a - 2 < GL || b + 2 > GH) {
                    const int32_t nGL = a - 2 < GL ? max(a - 2 - 30, -rlen - 2) : GL;
                    const int32_t nGH = b + 2 > GH ? min(b + 2 + 30, qlen + 2) : GH;
                    for (int sl = 0; sl < nslot; ++sl) {
                        int32_t *rowp = base + (int64_t)sl * slot_width;
                        for (int32_t k = nGL + lane; k < GL; k += 32)
                            rowp[k] = WFA_NEG_C;
                        for (int32_t k = GH + 1 + lane; k <= nGH; k += 32)
                            rowp[k] = WFA_NEG_C;
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
            __syncwarp();
            if (__any_sync(FULL, hit))
                result = s;
        }
        __syncwarp();  // the record is complete and visible to lane 0
        if (lane != 0)
            continue;
        if (overrun || result != c) {  // the cost pass and this pass disagree
            atomicOr(err_flag, 2);
            run_count[pi] = -1;
            continue;
        }
        // traceback by lane 0 (ops back to front, merged into runs)
        const Hist h{rec, hdr};
        uint32_t *const dst = runs + run_off[pi];
        const int64_t cap = (int64_t)qlen + rlen + 1;
        int64_t nrun = 0;
        uint32_t cur_op = 4, cur_len = 0;
        bool bad = false;
        auto emit = [&](uint32_t op, int32_t cnt) {
            if (cnt <= 0)
                return;
            if (op == cur_op) {
                cur_len += (uint32_t)cnt;
                return;
            }
            if (cur_len) {
                if (nrun >= cap) {
                    bad = true;
                    return;
                }
                dst[nrun++] = cur_len << 2 | cur_op;
            }
            cur_op = op;
            cur_len = (uint32_t)cnt;
        };
        int sp = c / g, mode = 0;
        int32_t k = target, crow = h.mafter(sp, k);
        for (int64_t guard = 4 * ((int64_t)qlen + rlen) + 16; !bad; --guard) {
            if (guard <= 0 || sp < 0) {
                bad = true;
                break;
            }
            if (mode == 0) {
                const uint32_t src = h.dec(sp, k) & 3u;
                int32_t before;
                if (sp == 0) {
                    before = 0;  // M[0, 0] = 0 before extension
                } else if (src == 1) {
                    before = h.mafter(sp - xs, k) + 1;
                } else if (src == 2) {
                    int ssp = sp, j = 0;
                    int32_t kk = k;
                    while (ssp >= 0 && (h.dec(ssp, kk) & 4u)) {
                        ssp -= es;
                        kk -= 1;
                        ++j;
                    }
                    before = h.mafter(ssp - oes, kk - 1) + 1 + j;
                } else if (src == 3) {
                    int ssp = sp;
                    int32_t kk = k;
                    while (ssp >= 0 && (h.dec(ssp, kk) & 8u)) {
                        ssp -= es;
                        kk += 1;
                    }
                    before = h.mafter(ssp - oes, kk + 1);
                } else {
                    bad = true;
                    break;
                }
                emit(0, crow - before);
                crow = before;
                if (sp == 0) {
                    if (k != 0)
                        bad = true;
                    break;
                }
                if (src == 1) {
                    emit(1, 1);
                    sp -= xs;
                    crow = h.mafter(sp, k);
                } else {
                    mode = (int)src - 1;  // 1: I, 2: D
                }
            } else if (mode == 1) {
                emit(2, 1);
                if (h.dec(sp, k) & 4u) {
                    sp -= es;
                    k -= 1;
                    crow -= 1;
                } else {
                    sp -= oes;
                    k -= 1;
                    crow = h.mafter(sp, k);
                    mode = 0;
                }
            } else {
                emit(3, 1);
                if (h.dec(sp, k) & 8u) {
                    sp -= es;
                    k += 1;
                } else {
                    sp -= oes;
                    k += 1;
                    crow = h.mafter(sp, k);
                    mode = 0;
                }
            }
        }
        if (!bad && cur_len) {
            if (nrun >= cap)
                bad = true;
            else
                dst[nrun++] = cur_len << 2 | cur_op;
        }
        if (bad) {
            atomicOr(err_flag, 4);
            run_count[pi] = -1;
            continue;
        }
        for (int64_t i = 0, j = nrun - 1; i < j; ++i, --j) {
            const uint32_t t = dst[i];
            dst[i] = dst[j];
            dst[j] = t;
        }
        run_count[pi] = (int32_t)nrun;
    }
}

// Gathers every pair's runs into one contiguous array (warp per pair).
__global__ void k_compact_runs(int64_t n, const uint32_t *__restrict__ runs,
                               const int64_t *__restrict__ run_off,
                               const int32_t *__restrict__ run_count,
                               const int64_t *__restrict__ out_off, uint32_t *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = w0; i < n; i += nw) {
        const int32_t m = run_count[i];
        for (int32_t j = lane; j < m; j += 32)
            out[out_off[i] + j] = runs[run_off[i] + j];
    }
}

}  // namespace

cudaError_t launch_wfa_cigar(SeqView q, SeqView r, WfaParams p, const int32_t *pairs, int64_t n,
                             int *counter, const int32_t *cost, const int64_t *hist_cells,
                             const int64_t *arena_off, uint8_t *arena, int32_t *scratch,
                             int64_t slot_width, int grid, uint32_t *runs,
                             const int64_t *run_off, int32_t *run_count, int *err_flag,
                             cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    wfa_cigar_kernel<<<grid, 128, 0, st>>>(q, r, p, pairs, n, counter, cost, hist_cells,
                                           arena_off, arena, scratch, slot_width, runs, run_off,
                                           run_count, err_flag);
    return cudaGetLastError();
}

static int cigar_blocks_per_sm()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, wfa_cigar_kernel, 128, 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    return std::max(nb, 1);
}

}  // namespace gb2

using namespace gb2;

// Host side of gb2_wfa_cigar: the cost pass, then the CIGAR pass in groups of
// pairs whose history records fit the arena budget, then the runs gathered.
static int wfa_cigar_run(gb2_ctx *c, SeqView qv, SeqView rv, const int64_t *h_qlen,
                         const int64_t *h_rlen, int64_t qmax, int64_t rmax,
                         const gb2_wfa_cfg *cfg, int64_t n, int32_t *cost, uint32_t *runs,
                         int64_t runs_cap, int64_t *run_offsets, int flags)
{
    Exec &x = c->x;
    CigarBufs &cb = c->cig;
    int rc;
    if ((rc = wfa_begin(c, x)) || (rc = ensure(c, cb.cost, (size_t)n * 4, x.st)) ||
        (rc = ensure(c, cb.hist, (size_t)n * 8, x.st)))
        return rc;
    if ((rc = wfa_core(c, x, qv, rv, qmax, rmax, cfg, n, (int32_t *)cb.cost.p,
                       flags | GB2_FLAG_BATCHED, (int64_t *)cb.hist.p)))
        return rc;
    if ((rc = wfa_end(c, x)))
        return rc;
    std::vector<int64_t> hist((size_t)n);
    GB2_CU(c, cudaMemcpyAsync(cost, cb.cost.p, (size_t)n * 4, cudaMemcpyDeviceToHost, x.st));
    GB2_CU(c, cudaMemcpyAsync(hist.data(), cb.hist.p, (size_t)n * 8, cudaMemcpyDeviceToHost,
                              x.st));
    GB2_CU(c, cudaStreamSynchronize(x.st));

    const int g = std::gcd(cfg->x, std::gcd(cfg->o, cfg->e));
    // per pair: record bytes, run capacity and its offset
    std::vector<int64_t> rec((size_t)n), run_off((size_t)n);
    int64_t run_total = 0, rec_max = 0;
    std::vector<int32_t> order;
    order.reserve((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        run_off[(size_t)i] = run_total;
        run_total += h_qlen[i] + h_rlen[i] + 1;
        rec[(size_t)i] = 0;
        if (cost[i] > 0 || (cost[i] == 0 && (h_qlen[i] | h_rlen[i]))) {
            rec[(size_t)i] = wfa_hist_record_bytes(hist[(size_t)i], cost[i] / g + 1);
            rec_max = std::max(rec_max, rec[(size_t)i]);
        }
        order.push_back((int32_t)i);
    }
    // largest records first: they carry the longest dependency chains
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return rec[(size_t)a] > rec[(size_t)b]; });
    size_t free_b = 0, total_b = 0;
    GB2_CU(c, cudaMemGetInfo(&free_b, &total_b));
    int64_t budget = std::min<int64_t>((int64_t)free_b / 2, kCigarArenaCap);
    if (rec_max >= (1ll << 33))  // header offsets are int32 counts of 4-byte words
        return set_err(c, GB2_ERANGE, "one pair's WFA history needs %lld bytes (limit 8 GiB)",
                       (long long)rec_max);
    if (rec_max > budget)
        return set_err(c, GB2_ENOMEM, "one pair's WFA history needs %lld bytes, %lld available",
                       (long long)rec_max, (long long)budget);

    const WfaParams p{cfg->x, cfg->o, cfg->e, cfg->max_error};
    const int hm = std::max(cfg->x / g, (cfg->o + cfg->e) / g) + 1, hie = cfg->e / g + 1;
    const int nslot = hm + 2 * hie;
    const int64_t slot_width = ((qmax + rmax + 5) + 31) & ~int64_t(31);
    const int64_t warp_bytes = (int64_t)nslot * slot_width * 4;
    int64_t grid = (int64_t)c->sm_count * cigar_blocks_per_sm();
    grid = std::min(grid, std::max<int64_t>(c->sm_count, kWfaScratchCap / (4 * warp_bytes)));
    grid = std::min(grid, std::max<int64_t>(1, (n + 3) / 4));
    // the arena: the budget, or all records when they fit in less
    int64_t all_rec = 0;
    for (int64_t i = 0; i < n; ++i)
        all_rec += rec[(size_t)i];
    const int64_t arena_bytes = std::max<int64_t>(16, std::min(budget, all_rec));
    if ((rc = ensure(c, x.scratch32, (size_t)(grid * 4 * warp_bytes), x.st)) ||
        (rc = ensure(c, x.counters, 4096, x.st)) ||
        (rc = ensure(c, cb.arena, (size_t)arena_bytes, x.st)) ||
        (rc = ensure(c, cb.pairs, (size_t)n * 4, x.st)) ||
        (rc = ensure(c, cb.arena_off, (size_t)n * 8, x.st)) ||
        (rc = ensure(c, cb.runs, (size_t)std::max<int64_t>(run_total, 1) * 4, x.st)) ||
        (rc = ensure(c, cb.run_off, (size_t)n * 8, x.st)) ||
        (rc = ensure(c, cb.run_count, (size_t)n * 4, x.st)) ||
        (rc = ensure(c, cb.out_off, (size_t)n * 8, x.st)) ||
        (rc = ensure(c, cb.out, (size_t)std::max<int64_t>(run_total, 1) * 4, x.st)))
        return rc;
    GB2_CU(c, cudaMemcpyAsync(cb.run_off.p, run_off.data(), (size_t)n * 8,
                              cudaMemcpyHostToDevice, x.st));
    GB2_CU(c, cudaMemsetAsync(cb.run_count.p, 0, (size_t)n * 4, x.st));
    // groups of pairs (largest first) whose records fit the arena together
    std::vector<int64_t> aoff((size_t)n, 0);
    for (size_t g0 = 0; g0 < order.size();) {
        size_t g1 = g0;
        int64_t used = 0;
        while (g1 < order.size() && used + rec[(size_t)order[g1]] <= arena_bytes) {
            aoff[(size_t)order[g1]] = used;
            used += rec[(size_t)order[g1]];
            ++g1;
        }
        if (g1 == g0)  // cannot happen: every record fits the arena alone
            return set_err(c, GB2_ENOMEM, "WFA history arena too small");
        const int64_t m = (int64_t)(g1 - g0);
        GB2_CU(c, cudaMemcpyAsync(cb.pairs.p, order.data() + g0, (size_t)m * 4,
                                  cudaMemcpyHostToDevice, x.st));
        GB2_CU(c, cudaMemcpyAsync(cb.arena_off.p, aoff.data(), (size_t)n * 8,
                                  cudaMemcpyHostToDevice, x.st));
        GB2_CU(c, cudaMemsetAsync(x.counters.p, 0, 64, x.st));
        GB2_CU(c, launch_wfa_cigar(qv, rv, p, (const int32_t *)cb.pairs.p, m,
                                   (int *)x.counters.p, (const int32_t *)cb.cost.p,
                                   (const int64_t *)cb.hist.p,
                                   (const int64_t *)cb.arena_off.p, (uint8_t *)cb.arena.p,
                                   (int32_t *)x.scratch32.p, slot_width,
                                   (int)std::min<int64_t>(grid, (m + 3) / 4),
                                   (uint32_t *)cb.runs.p, (const int64_t *)cb.run_off.p,
                                   (int32_t *)cb.run_count.p, (int *)x.errflag.p, x.st));
        c->launches += 1;
        // the host arrays of this group stay untouched until its copies are done
        GB2_CU(c, cudaStreamSynchronize(x.st));
        g0 = g1;
    }
    int flag = 0;
    std::vector<int32_t> cnt((size_t)n);
    GB2_CU(c, cudaMemcpyAsync(&flag, x.errflag.p, 4, cudaMemcpyDeviceToHost, x.st));
    GB2_CU(c, cudaMemcpyAsync(cnt.data(), cb.run_count.p, (size_t)n * 4, cudaMemcpyDeviceToHost,
                              x.st));
    GB2_CU(c, cudaStreamSynchronize(x.st));
    if (flag)
        return set_err(c, GB2_EKERNEL, "WFA CIGAR kernel reported error bits %d", flag);
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) {
        run_offsets[i] = total;
        total += cnt[(size_t)i];
    }
    run_offsets[n] = total;
    if (total > runs_cap)
        return set_err(c, GB2_ERANGE, "CIGAR runs need %lld entries, runs_cap is %lld",
                       (long long)total, (long long)runs_cap);
    if (total == 0)
        return GB2_OK;
    GB2_CU(c, cudaMemcpyAsync(cb.out_off.p, run_offsets, (size_t)n * 8, cudaMemcpyHostToDevice,
                              x.st));
    const int blocks = (int)std::min<int64_t>((n + 3) / 4, (int64_t)c->sm_count * 16);
    k_compact_runs<<<blocks, 128, 0, x.st>>>(n, (const uint32_t *)cb.runs.p,
                                             (const int64_t *)cb.run_off.p,
                                             (const int32_t *)cb.run_count.p,
                                             (const int64_t *)cb.out_off.p, (uint32_t *)cb.out.p);
    GB2_CU(c, cudaGetLastError());
    c->launches += 1;
    GB2_CU(c, cudaMemcpyAsync(runs, cb.out.p, (size_t)total * 4, cudaMemcpyDeviceToHost, x.st));
    GB2_CU(c, cudaStreamSynchronize(x.st));
    return GB2_OK;
}

extern "C" {

int gb2_wfa_cigar(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_wfa_cfg *cfg,
                  int64_t n, int32_t *cost, uint32_t *runs, int64_t runs_cap,
                  int64_t *run_offsets, int flags)
{
    if (!c || !q || !r)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (q->owner != c || r->owner != c)
        return set_err(c, GB2_EINVAL, "batch belongs to another context");
    if (n > q->count || n > r->count)
        return set_err(c, GB2_EINVAL, "n_pairs exceeds a batch's sequence count");
    int rc = wfa_validate(c, cfg, n);
    if (rc)
        return rc;
    if (!run_offsets || (n > 0 && (!cost || (runs_cap > 0 && !runs))) || runs_cap < 0)
        return set_err(c, GB2_EINVAL, "cost, runs or run_offsets missing");
    run_offsets[0] = 0;
    if (n == 0)
        return GB2_OK;
    std::vector<int64_t> ql((size_t)n), rl((size_t)n);
    GB2_CU(c, cudaMemcpyAsync(ql.data(), q->d_lengths, (size_t)n * 8, cudaMemcpyDeviceToHost,
                              c->x.st));
    GB2_CU(c, cudaMemcpyAsync(rl.data(), r->d_lengths, (size_t)n * 8, cudaMemcpyDeviceToHost,
                              c->x.st));
    GB2_CU(c, cudaStreamSynchronize(c->x.st));
    const SeqView qv{q->d_packed, q->d_offsets, q->d_lengths, 0, q->n_words};
    const SeqView rv{r->d_packed, r->d_offsets, r->d_lengths, 0, r->n_words};
    return wfa_cigar_run(c, qv, rv, ql.data(), rl.data(), q->max_len, r->max_len, cfg, n, cost,
                         runs, runs_cap, run_offsets, flags);
}

int gb2_wfa_cigar_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen,
                       const uint64_t *r_words, int64_t rlen, const gb2_wfa_cfg *cfg,
                       int32_t *cost, char *cigar, int64_t cap)
{
    if (!c || !cost || !cigar || cap < 1 || qlen < 0 || rlen < 0 ||
        (qlen > 0 && !q_words) || (rlen > 0 && !r_words))
        return GB2_EINVAL;
    cigar[0] = 0;
    const int64_t qn = words_for(qlen), rn = words_for(rlen);
    const int64_t zero = 0;
    gb2_batch *qb = nullptr, *rb = nullptr;
    const uint64_t pad = 0;
    int rc = gb2_batch_upload(c, qn ? q_words : &pad, std::max<int64_t>(qn, 1), nullptr, &zero,
                              &qlen, 1, &qb);
    if (!rc)
        rc = gb2_batch_upload(c, rn ? r_words : &pad, std::max<int64_t>(rn, 1), nullptr, &zero,
                              &rlen, 1, &rb);
    std::vector<uint32_t> runs((size_t)(qlen + rlen + 1));
    int64_t off[2] = {0, 0};
    if (!rc)
        rc = gb2_wfa_cigar(c, qb, rb, cfg, 1, cost, runs.data(), (int64_t)runs.size(), off, 0);
    gb2_batch_free(c, qb);
    gb2_batch_free(c, rb);
    if (rc)
        return rc;
    static const char opc[4] = {'=', 'X', 'I', 'D'};
    int64_t pos = 0;
    for (int64_t i = off[0]; i < off[1]; ++i) {
        char buf[24];
        const int len = snprintf(buf, sizeof buf, "%u%c", runs[(size_t)i] >> 2,
                                 opc[runs[(size_t)i] & 3u]);
        if (pos + len + 1 > cap) {
            cigar[0] = 0;
            return GB2_ERANGE;
        }
        memcpy(cigar + pos, buf, (size_t)len);
        pos += len;
    }
    cigar[pos] = 0;
    return GB2_OK;
}

}  // extern "C"
