// nw.cu -- banded Needleman-Wunsch (global) on sm_100a.
//
// needleman_wunsch_banded (genomics/cpu/align_cpu.mojo:312-377) with its
// intended semantics: the reference creates the two band rows with capacity
// only and indexes them (:327-341); here, as in the oracle, both rows have
// 2*band+1 elements, and every other statement is the reference's:
//   initial row: column ri = j - band holds NEG (-1,000,000) for ri < 0, 0
//     for ri = 0, gap_open + ri*gap_extend otherwise (:330-337);
//   row qi: every cell starts at NEG; cells with ri = qi - band + j inside
//     [0, rlen) get max(H_diag + sub, H_up + go + ge, H_left + go + ge) where
//     H_diag = prev[j], H_up = prev[j+1] (NEG past the band), H_left = cur[j-1]
//     (NEG at j = 0) (:342-362);
//   score = prev[(rlen-1) - (qlen-1) + band] when inside the band, else NEG;
//   query_end = qlen - 1, ref_end = rlen - 1 (:365-376).
// NEG is an ordinary number in this recurrence (it is added to), so every
// value is reproduced exactly: int32 in the register kernel when the host has
// checked that no value can leave int32, int64 in the literal kernel.
//
// nw_band_kernel<B> (B = 16, 32): one thread per pair, the band row in
// 2B+1 registers updated in place left to right (a cell reads the old value of
// its own and its right neighbour's register and the new value of its left
// one).  Substitution scores come from per-row equality bits: the reference
// window's 2-bit codes XOR the replicated query base, folded to one bit per
// base.  Rows with no cell left of the reference start skip the masking
// (cells past the reference end feed no cell inside the matrix).
// nw_literal_kernel: one thread per pair, int64 rows in global scratch, any
// band, per-pair bands.
#include <algorithm>

#include "runtime.cuh"

namespace gb2 {
namespace {

constexpr int64_t kNwNeg = -1000000;

template <int B, bool MASK>
__device__ __forceinline__ void nw_row(int32_t (&H)[2 * B + 1], const uint64_t *eqc, int lo,
                                       int hi, int32_t match, int32_t mismatch, int32_t goe)
{
    constexpr int W = 2 * B + 1;
    const int32_t dm = match - mismatch;
    int32_t left = (int32_t)kNwNeg;
#pragma unroll
    for (int j = 0; j < W; ++j) {
        const int32_t bit = (int32_t)((eqc[j >> 5] >> (62 - 2 * (j & 31))) & 1u);
        const int32_t sub = mismatch + bit * dm;
        const int32_t up = (j + 1 < W) ? H[j + 1 < W ? j + 1 : j] : (int32_t)kNwNeg;
        int32_t cell = max(H[j] + sub, max(up, left) + goe);
        if (MASK && (j < lo || j >= hi))
            cell = (int32_t)kNwNeg;
        H[j] = cell;
        left = cell;
    }
}

template <int B>
__global__ void __launch_bounds__(128)
nw_band_kernel(SeqView q, SeqView r, SwParams p, int64_t n, int *counter,
               gb2_sw_result *__restrict__ out)
{
    constexpr int W = 2 * B + 1;
    constexpr int NWIN = (W + 31) / 32;
    const int lane = threadIdx.x & 31;
    const int32_t goe = p.go + p.ge;
    for (;;) {
        int64_t b0 = 0;
        if (lane == 0)
            b0 = atomicAdd(counter, 32);
        const int64_t base = __shfl_sync(0xffffffffu, b0, 0);
        if (base >= n)
            break;
        const int64_t pi = base + lane;
        if (pi >= n)
            continue;
        const int64_t qoff = q.offsets[pi] - q.word_base;
        const int64_t roff = r.offsets[pi] - r.word_base;
        const int32_t qlen = (int32_t)q.lengths[pi], rlen = (int32_t)r.lengths[pi];
        int32_t H[W];
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const int ri = j - B;
            H[j] = ri < 0 ? (int32_t)kNwNeg : (ri == 0 ? 0 : p.go + ri * p.ge);
        }
        for (int32_t qi = 0; qi < qlen; ++qi) {
            const uint64_t qw = __ldg(q.packed + qoff + (qi >> 5));
            const uint64_t qrep = ((qw >> (62 - 2 * (qi & 31))) & 3u) * 0x5555555555555555ull;
            const int64_t ri0 = (int64_t)qi - B;
            const int64_t w = roff + (ri0 >> 5);
            const int sh = (int)(ri0 & 31) * 2;
            uint64_t words[NWIN + 1], eqc[NWIN];
#pragma unroll
            for (int i = 0; i <= NWIN; ++i) {
                int64_t wi = w + i;
                wi = wi < 0 ? 0 : (wi >= r.n_words ? r.n_words - 1 : wi);
                words[i] = __ldg(r.packed + wi);
            }
#pragma unroll
            for (int i = 0; i < NWIN; ++i) {
                const uint64_t win = sh ? ((words[i] << sh) | (words[i + 1] >> (64 - sh))) : words[i];
                const uint64_t x = win ^ qrep;
                eqc[i] = ~(x | (x >> 1)) & 0x5555555555555555ull;
            }
            // cells j with ri = qi - B + j in [0, rlen).  Cells past the reference
            // end (ri >= rlen) need not be NEG: no cell inside the matrix reads
            // them (diag, up and left of a cell all have ri' <= its ri) and the
            // score is read inside the matrix, so only rows that reach left of
            // the reference start take the masked step
            const int lo = max(0, B - qi);
            const int hi = (int)min((int64_t)W, (int64_t)B - qi + rlen);
            if (lo == 0)
                nw_row<B, false>(H, eqc, lo, hi, p.match, p.mismatch, goe);
            else
                nw_row<B, true>(H, eqc, lo, hi, p.match, p.mismatch, goe);
        }
        const int64_t fo = (int64_t)(rlen - 1) - (qlen - 1) + B;
        int32_t score = (int32_t)kNwNeg;
#pragma unroll
        for (int j = 0; j < W; ++j)
            if (fo == j)
                score = H[j];
        gb2_sw_result res;
        res.score = score;
        res.query_end = qlen - 1;
        res.ref_end = rlen - 1;
        out[pi] = res;
    }
}

__global__ void __launch_bounds__(128)
nw_literal_kernel(SeqView q, SeqView r, SwParams p, int32_t band, const int32_t *__restrict__ bands,
                  int64_t n, gb2_sw_result *__restrict__ out, int64_t *__restrict__ scratch,
                  int64_t stride)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    int64_t *hp = scratch + tid * stride;
    for (int64_t pi = tid; pi < n; pi += nth) {
        const int64_t b = bands ? bands[pi] : band;
        const int64_t width = 2 * b + 1;
        int64_t *hc = hp + width;
        const int64_t qlen = q.lengths[pi], rlen = r.lengths[pi];
        const uint64_t *qw = q.packed + (q.offsets[pi] - q.word_base);
        const uint64_t *rw = r.packed + (r.offsets[pi] - r.word_base);
        for (int64_t j = 0; j < width; ++j) {
            const int64_t ri = -b + j;
            hp[j] = ri < 0 ? kNwNeg : (ri == 0 ? 0 : p.go + ri * p.ge);
        }
        for (int64_t qi = 0; qi < qlen; ++qi) {
            for (int64_t j = 0; j < width; ++j)
                hc[j] = kNwNeg;
            const int64_t qb = (int64_t)((qw[qi >> 5] >> (62 - 2 * (qi & 31))) & 3u);
            for (int64_t off = 0; off < width; ++off) {
                const int64_t ri = qi - b + off;
                if (ri < 0 || ri >= rlen)
                    continue;
                const int64_t rb = (int64_t)((rw[ri >> 5] >> (62 - 2 * (ri & 31))) & 3u);
                const int64_t sub = (qb == rb) ? p.match : p.mismatch;
                const int64_t h_diag = hp[off];
                const int64_t h_up = (off + 1 < width) ? hp[off + 1] : kNwNeg;
                const int64_t h_left = (off > 0) ? hc[off - 1] : kNwNeg;
                int64_t cell = h_diag + sub;
                const int64_t e = h_up + p.go + p.ge, f = h_left + p.go + p.ge;
                cell = cell > e ? cell : e;
                cell = cell > f ? cell : f;
                hc[off] = cell;
            }
            for (int64_t j = 0; j < width; ++j)
                hp[j] = hc[j];
        }
        const int64_t fo = (rlen - 1) - (qlen - 1) + b;
        gb2_sw_result res;
        res.score = (int32_t)((fo >= 0 && fo < width) ? hp[fo] : kNwNeg);
        res.query_end = (int32_t)(qlen - 1);
        res.ref_end = (int32_t)(rlen - 1);
        out[pi] = res;
    }
}

template <int B>
int nw_blocks_per_sm()
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, nw_band_kernel<B>, 128, 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    return std::max(nb, 1);
}

}  // namespace
}  // namespace gb2

using namespace gb2;

// Runs NW over n resident pairs into d_out (device); blocking.
static int nw_core(gb2_ctx *c, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
                   const gb2_sw_cfg *cfg, const int32_t *h_bands, int64_t n,
                   gb2_sw_result *d_out, int flags)
{
    if (!cfg)
        return set_err(c, GB2_EINVAL, "cfg is NULL");
    int64_t maxb = cfg->band_width;
    if (h_bands) {
        maxb = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (h_bands[i] < 0)
                return set_err(c, GB2_EINVAL, "band of pair %lld is negative", (long long)i);
            maxb = std::max<int64_t>(maxb, h_bands[i]);
        }
    } else if (cfg->band_width < 0) {
        return set_err(c, GB2_EINVAL, "band_width < 0");
    }
    // every value of the recurrence stays within NEG - pmax*(qlen + rlen + 2b + 2) and
    // pmax*(qlen + rlen + 2b + 2); int32 results need that inside int32
    const int64_t pmax = std::abs((int64_t)cfg->match_score) + std::abs((int64_t)cfg->mismatch) +
                         std::abs((int64_t)cfg->gap_open) + std::abs((int64_t)cfg->gap_extend);
    if (qmax >= (1ll << 30) || rmax >= (1ll << 30) ||
        -kNwNeg + pmax * (qmax + rmax + 2 * maxb + 2) >= (1ll << 31))
        return set_err(c, GB2_ERANGE, "NW values could leave the int32 range");
    Exec &x = c->x;
    const SwParams p{cfg->match_score, cfg->mismatch, cfg->gap_open, cfg->gap_extend};
    const int32_t band = cfg->band_width;
    const bool reg = !h_bands && (band == 16 || band == 32) && !(flags & GB2_FLAG_GENERIC);
    if (reg) {
        int rc;
        if ((rc = ensure(c, x.counters, 4096, x.st)))
            return rc;
        GB2_CU(c, cudaMemsetAsync(x.counters.p, 0, 64, x.st));
        const int per = band == 16 ? nw_blocks_per_sm<16>() : nw_blocks_per_sm<32>();
        const int grid = (int)std::min<int64_t>((int64_t)c->sm_count * per, (n + 127) / 128);
        if (band == 16)
            nw_band_kernel<16><<<grid, 128, 0, x.st>>>(qv, rv, p, n, (int *)x.counters.p, d_out);
        else
            nw_band_kernel<32><<<grid, 128, 0, x.st>>>(qv, rv, p, n, (int *)x.counters.p, d_out);
        GB2_CU(c, cudaGetLastError());
    } else {
        const int32_t *d_bands = nullptr;
        int rc;
        if (h_bands) {
            if ((rc = ensure(c, c->bands, (size_t)n * 4, x.st)) || (rc = h2d(c, c->bands.p, h_bands, (size_t)n * 4, x.st)))
                return rc;
            d_bands = (const int32_t *)c->bands.p;
        }
        const int64_t stride = 2 * (2 * maxb + 1);
        const int grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)c->sm_count * 4);
        if ((rc = ensure(c, x.scratch64, (size_t)grid * 128 * stride * 8, x.st)))
            return rc;
        nw_literal_kernel<<<grid, 128, 0, x.st>>>(qv, rv, p, band, d_bands, n, d_out,
                                                  (int64_t *)x.scratch64.p, stride);
        GB2_CU(c, cudaGetLastError());
    }
    c->launches += 1;
    return GB2_OK;
}

extern "C" {

static int gb2_nw_banded_impl(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_sw_cfg *cfg,
                  const int32_t *bands, int64_t n, gb2_sw_result *out, int flags)
{
    if (!c || !q || !r)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (q->owner != c || r->owner != c)
        return set_err(c, GB2_EINVAL, "batch belongs to another context");
    if (n < 0 || n > q->count || n > r->count)
        return set_err(c, GB2_EINVAL, "n_pairs outside the batches' sequence counts");
    if (n > 0 && !out)
        return set_err(c, GB2_EINVAL, "out is NULL");
    if (n == 0)
        return cfg ? GB2_OK : set_err(c, GB2_EINVAL, "cfg is NULL");
    int rc;
    if ((rc = ensure(c, c->out_sw, (size_t)n * sizeof(gb2_sw_result), c->x.st)))
        return rc;
    const SeqView qv{q->d_packed, q->d_offsets, q->d_lengths, 0, q->n_words};
    const SeqView rv{r->d_packed, r->d_offsets, r->d_lengths, 0, r->n_words};
    if ((rc = nw_core(c, qv, rv, q->max_len, r->max_len, cfg, bands, n,
                      (gb2_sw_result *)c->out_sw.p, flags)))
        return rc;
    GB2_CU(c, cudaMemcpyAsync(out, c->out_sw.p, (size_t)n * sizeof(gb2_sw_result),
                              cudaMemcpyDeviceToHost, c->x.st));
    GB2_CU(c, cudaStreamSynchronize(c->x.st));
    return GB2_OK;
}

int gb2_nw_banded(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_sw_cfg *cfg,
                  const int32_t *bands, int64_t n, gb2_sw_result *out, int flags)
{
    return drain_on_error(c, gb2_nw_banded_impl(c, q, r, cfg, bands, n, out, flags));
}

static int gb2_nw_pair_impl(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                int64_t rlen, const gb2_sw_cfg *cfg, gb2_sw_result *out)
{
    if (!c || !out || qlen < 0 || rlen < 0 || (qlen > 0 && !q_words) || (rlen > 0 && !r_words))
        return GB2_EINVAL;
    const int64_t qn = words_for(qlen), rn = words_for(rlen);
    const int64_t zero = 0;
    const uint64_t pad = 0;
    gb2_batch *qb = nullptr, *rb = nullptr;
    int rc = gb2_batch_upload(c, qn ? q_words : &pad, std::max<int64_t>(qn, 1), nullptr, &zero,
                              &qlen, 1, &qb);
    if (!rc)
        rc = gb2_batch_upload(c, rn ? r_words : &pad, std::max<int64_t>(rn, 1), nullptr, &zero,
                              &rlen, 1, &rb);
    if (!rc)
        rc = gb2_nw_banded(c, qb, rb, cfg, nullptr, 1, out, 0);
    gb2_batch_free(c, qb);
    gb2_batch_free(c, rb);
    return rc;
}

int gb2_nw_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                int64_t rlen, const gb2_sw_cfg *cfg, gb2_sw_result *out)
{
    return drain_on_error(c, gb2_nw_pair_impl(c, q_words, qlen, r_words, rlen, cfg, out));
}

}  // extern "C"
