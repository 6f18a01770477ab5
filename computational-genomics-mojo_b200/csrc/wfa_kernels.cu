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
//  * NEG is a large negative number and sources are combined with plain max:
//    a NEG source plus at most one per score stays negative, and every
//    non-NEG value is >= 0, so "negative" reproduces the reference's
//    "== NEG_INF" tests (:174-204) and its "row < 0" skip (:211).
//
// One warp aligns one pair.  Ring slots live in a per-warp scratch region,
// one int32 per diagonal (index k + rlen + 2).  Invariant: inside the
// interval [GL, GH] that this pair has touched (every visited interval
// widened by 2), every slot position outside that slot's own interval holds
// NEG; so source reads at k-1, k, k+1 need no bounds tests.
#include "gb2_internal.cuh"

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

// Extend (align_cpu.mojo:208-219), 32 bases per step: XOR of the two
// unaligned 64-bit windows, count leading zeros, clamp by the remaining
// lengths (zero padding past a sequence end decodes as A).
__device__ __forceinline__ int32_t wfa_extend(const SeqView &q, int64_t qoff, int32_t qlen,
                                              const SeqView &r, int64_t roff, int32_t rlen,
                                              int32_t row, int32_t k)
{
    int32_t col = row - k;
    if (row < 0 || col < 0)
        return row;
    while (row < qlen && col < rlen) {
        const uint64_t a = load_window64(q.packed, q.n_words, qoff, row);
        const uint64_t b = load_window64(r.packed, r.n_words, roff, col);
        const uint64_t x = a ^ b;
        const int ml = x ? (__clzll((long long)x) >> 1) : 32;
        const int lim = min(qlen - row, rlen - col);
        if (ml >= lim) {
            row += lim;
            col += lim;
            break;
        }
        row += ml;
        col += ml;
        if (ml < 32)
            break;
    }
    return row;
}

__global__ void __launch_bounds__(128)
wfa_warp_kernel(SeqView q, SeqView r, WfaParams p, PairList pl, int32_t *__restrict__ out,
                int32_t *__restrict__ scratch, int64_t slot_width, int *err_flag, int64_t *work)
{
    int64_t n;
    const int32_t *__restrict__ queue = pairs_resolve(pl, n);
    int *const queue_counter = pl.counter;
    const int lane = threadIdx.x & 31;
    const int64_t warp_global = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);
    const unsigned FULL = 0xffffffffu;

    const int g = gcd_i(p.x, gcd_i(p.o, p.e));
    const int xs = p.x / g, oes = (p.o + p.e) / g, es = p.e / g;
    const int hm = max(xs, oes) + 1, hie = es + 1;
    const int nslot = hm + 2 * hie;
    int32_t *const region = scratch + warp_global * nslot * slot_width;
    const int64_t max_err = p.max_error;

    int64_t next = warp_global;
    for (;;) {
        int64_t slot_i = next;
        if (queue_counter) {
            int64_t b0 = 0;
            if (lane == 0)
                b0 = atomicAdd(queue_counter, 1);
            slot_i = __shfl_sync(FULL, b0, 0);
        }
        if (slot_i >= n)
            break;
        next += warps_total;
        const int64_t pi = queue ? (int64_t)queue[slot_i] : slot_i;
        const int64_t qoff = q.offsets[pi] - q.word_base;
        const int64_t roff = r.offsets[pi] - r.word_base;
        const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
        int32_t result = -1;
        int64_t cells = 0;
        if (qlen == 0 && rlen == 0) {
            result = 0;
        } else if ((int64_t)qlen + rlen + 5 > slot_width) {
            if (lane == 0)
                atomicOr(err_flag, 1);
            result = -2;
        } else {
            const int32_t kofs = rlen + 2;
            const int32_t target = qlen - rlen;
            auto M = [&](int slot) { return region + (int64_t)slot * slot_width + kofs; };
            auto I = [&](int slot) { return region + (int64_t)(hm + slot) * slot_width + kofs; };
            auto D = [&](int slot) {
                return region + (int64_t)(hm + hie + slot) * slot_width + kofs;
            };
            // per-slot intervals: lane j holds slot j's (ring sizes <= 32)
            int32_t mlo = 1, mhi = 0, ilo = 1, ihi = 0, dlo = 1, dhi = 0;
            int32_t GL = max(-2, -rlen - 2), GH = min(2, qlen + 2);
            for (int sl = 0; sl < nslot; ++sl) {
                int32_t *row = region + (int64_t)sl * slot_width + kofs;
                for (int32_t k = GL + lane; k <= GH; k += 32)
                    row[k] = WFA_NEG;
            }
            __syncwarp();
            // score 0: M[0,0] = 0 extended along diagonal 0 (:130-140)
            int32_t row0 = 0;
            if (lane == 0) {
                row0 = wfa_extend(q, qoff, qlen, r, roff, rlen, 0, 0);
                M(0)[0] = row0;
            }
            row0 = __shfl_sync(FULL, row0, 0);
            if (lane == 0) {
                mlo = 0;
                mhi = 0;
            }
            __syncwarp();
            if (target == 0 && row0 >= qlen && max_err >= 0) {
                result = 0;
            } else {
                for (int64_t sp = 1; sp * g <= max_err; ++sp) {
                    const int64_t s = sp * g;
                    int64_t lo = max((int64_t)-rlen, -s), hi = min((int64_t)qlen, s);
                    if (target < lo || target > hi) {
                        lo = min(lo, (int64_t)target);
                        hi = max(hi, (int64_t)target);
                    }
                    lo = max(lo, -max_err);
                    hi = min(hi, max_err);
                    int32_t ulo = 0x7fffffff, uhi = -0x7fffffff;
                    const int sx = sp >= xs ? (int)((sp - xs) % hm) : -1;
                    const int soe = sp >= oes ? (int)((sp - oes) % hm) : -1;
                    const int se = sp >= es ? (int)((sp - es) % hie) : -1;
                    if (sx >= 0) {
                        const int32_t a0 = __shfl_sync(FULL, mlo, sx), b0 = __shfl_sync(FULL, mhi, sx);
                        if (a0 <= b0) {
                            ulo = min(ulo, a0);
                            uhi = max(uhi, b0);
                        }
                    }
                    if (soe >= 0) {
                        const int32_t a0 = __shfl_sync(FULL, mlo, soe), b0 = __shfl_sync(FULL, mhi, soe);
                        if (a0 <= b0) {
                            ulo = min(ulo, a0 - 1);
                            uhi = max(uhi, b0 + 1);
                        }
                    }
                    if (se >= 0) {
                        const int32_t a0 = __shfl_sync(FULL, ilo, se), b0 = __shfl_sync(FULL, ihi, se);
                        if (a0 <= b0) {
                            ulo = min(ulo, a0 + 1);
                            uhi = max(uhi, b0 + 1);
                        }
                        const int32_t a1 = __shfl_sync(FULL, dlo, se), b1 = __shfl_sync(FULL, dhi, se);
                        if (a1 <= b1) {
                            ulo = min(ulo, a1 - 1);
                            uhi = max(uhi, b1 - 1);
                        }
                    }
                    const int32_t a = (int32_t)max((int64_t)ulo, lo);
                    const int32_t b = (int32_t)min((int64_t)uhi, hi);
                    const int ms = (int)(sp % hm), is = (int)(sp % hie);
                    const int32_t omlo = __shfl_sync(FULL, mlo, ms), omhi = __shfl_sync(FULL, mhi, ms);
                    const int32_t oilo = __shfl_sync(FULL, ilo, is), oihi = __shfl_sync(FULL, ihi, is);
                    const int32_t odlo = __shfl_sync(FULL, dlo, is), odhi = __shfl_sync(FULL, dhi, is);
                    int32_t *Mw = M(ms), *Iw = I(is), *Dw = D(is);
                    if (a > b) {
                        // empty score: clear what the reused slots held
                        for (int32_t k = omlo + lane; k <= omhi; k += 32)
                            Mw[k] = WFA_NEG;
                        for (int32_t k = oilo + lane; k <= oihi; k += 32)
                            Iw[k] = WFA_NEG;
                        for (int32_t k = odlo + lane; k <= odhi; k += 32)
                            Dw[k] = WFA_NEG;
                        if (lane == ms) {
                            mlo = 1;
                            mhi = 0;
                        }
                        if (lane == is) {
                            ilo = dlo = 1;
                            ihi = dhi = 0;
                        }
                        __syncwarp();
                        continue;
                    }
                    cells += (int64_t)(b - a + 1);
                    // widen the touched interval to [a-2, b+2]
                    const int32_t nGL = max(min(GL, a - 2), -rlen - 2);
                    const int32_t nGH = min(max(GH, b + 2), qlen + 2);
                    if (nGL < GL || nGH > GH) {
                        for (int sl = 0; sl < nslot; ++sl) {
                            int32_t *rowp = region + (int64_t)sl * slot_width + kofs;
                            for (int32_t k = nGL + lane; k < GL; k += 32)
                                rowp[k] = WFA_NEG;
                            for (int32_t k = GH + 1 + lane; k <= nGH; k += 32)
                                rowp[k] = WFA_NEG;
                        }
                        GL = nGL;
                        GH = nGH;
                        __syncwarp();
                    }
                    const int32_t *Mx = sx >= 0 ? M(sx) : nullptr;
                    const int32_t *Moe = soe >= 0 ? M(soe) : nullptr;
                    const int32_t *Ie = se >= 0 ? I(se) : nullptr;
                    const int32_t *De = se >= 0 ? D(se) : nullptr;
                    for (int32_t k = a + lane; k <= b; k += 32) {
                        int32_t iv = WFA_NEG, dv = WFA_NEG, mv = WFA_NEG;
                        if (Moe) {
                            iv = Moe[k - 1];
                            dv = Moe[k + 1];
                        }
                        if (Ie) {
                            iv = max(iv, Ie[k - 1]);
                            dv = max(dv, De[k + 1]);
                        }
                        iv += 1;
                        if (Mx)
                            mv = Mx[k] + 1;
                        mv = max(mv, max(iv, dv));
                        Iw[k] = iv;
                        Dw[k] = dv;
                        Mw[k] = mv;
                    }
                    // old contents of the reused slots outside [a, b] -> NEG
                    for (int32_t k = omlo + lane; k <= omhi; k += 32)
                        if (k < a || k > b)
                            Mw[k] = WFA_NEG;
                    for (int32_t k = oilo + lane; k <= oihi; k += 32)
                        if (k < a || k > b)
                            Iw[k] = WFA_NEG;
                    for (int32_t k = odlo + lane; k <= odhi; k += 32)
                        if (k < a || k > b)
                            Dw[k] = WFA_NEG;
                    if (lane == ms) {
                        mlo = a;
                        mhi = b;
                    }
                    if (lane == is) {
                        ilo = dlo = a;
                        ihi = dhi = b;
                    }
                    // extend this lane's diagonals (the lane wrote them itself)
                    for (int32_t k = a + lane; k <= b; k += 32) {
                        const int32_t row = Mw[k];
                        if (row >= 0)
                            Mw[k] = wfa_extend(q, qoff, qlen, r, roff, rlen, row, k);
                    }
                    bool done = false;
                    if (target >= lo && target <= hi && target >= a && target <= b) {
                        const int owner = (target - a) & 31;
                        int32_t v = 0;
                        if (lane == owner)
                            v = Mw[target];
                        v = __shfl_sync(FULL, v, owner);
                        done = v >= qlen;
                    }
                    __syncwarp();
                    if (done) {
                        result = (int32_t)s;
                        break;
                    }
                }
            }
        }
        if (lane == 0) {
            out[pi] = result;
            if (work)
                atomicAdd((unsigned long long *)work, (unsigned long long)cells);
        }
    }
}

cudaError_t launch_wfa(int variant, SeqView q, SeqView r, WfaParams p, PairList pl, int32_t *out,
                       int32_t *scratch, int64_t slot_width, int grid, int *err_flag,
                       int64_t *work, cudaStream_t st)
{
    (void)variant;
    if (!pl.seg && pl.n <= 0)
        return cudaSuccess;
    wfa_warp_kernel<<<grid, 128, 0, st>>>(q, r, p, pl, out, scratch, slot_width, err_flag,
                                          work);
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
