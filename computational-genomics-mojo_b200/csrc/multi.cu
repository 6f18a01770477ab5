// multi.cu -- one caller's pair list over several devices.
//
// Pairs are independent (the reference gives each its own thread block,
// genomics/gpu/align_gpu.mojo:80, :295), so the list splits into contiguous
// slices with no exchange step: gb2_partition_pairs cuts it where the
// cumulative work reaches k/parts of the total, each context aligns its slice
// from the caller's host arrays (its own upload, its own device), and the
// results land in the caller's output array at the slice's offset -- input
// order, nothing to gather but the slices themselves.  Across processes (one
// per GPU) the same partition is computed by every rank and the slices are
// gathered by the caller's collective (genomics_b200.multi).
#include <thread>
#include <vector>

#include "runtime.cuh"

namespace {

// Work units of pair i: Smith-Waterman cells qlen * (2 * band + 1) (the
// reference's count, benchmarks/bench_alignment.mojo:51); for WFA the square
// of the longer length (the visited cells grow with the square of the cost,
// which grows with the length at a given divergence).  Plus a fixed share per
// pair for its launch-independent costs (lengths, result, scheduling).
inline double work_of(int kind, int64_t ql, int64_t rl, int64_t band)
{
    constexpr double kPerPair = 1024.0;
    if (kind == 1) {
        const double l = (double)(ql > rl ? ql : rl);
        return l * l + kPerPair;
    }
    return (double)ql * (2.0 * (double)band + 1.0) + kPerPair;
}

}  // namespace

extern "C" {

int gb2_partition_pairs(const int64_t *q_lengths, const int64_t *r_lengths, const int32_t *bands,
                        int32_t band, int kind, int64_t n, int n_parts, int64_t *bounds)
{
    if (!bounds || n < 0 || n_parts < 1 || (kind != 0 && kind != 1) ||
        (n > 0 && (!q_lengths || !r_lengths)))
        return GB2_EINVAL;
    double total = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t b = bands ? bands[i] : band;
        if (q_lengths[i] < 0 || r_lengths[i] < 0 || b < 0)
            return GB2_EINVAL;
        total += work_of(kind, q_lengths[i], r_lengths[i], b);
    }
    bounds[0] = 0;
    int k = 1;
    double acc = 0.0;
    for (int64_t i = 0; i < n && k < n_parts; ++i) {
        acc += work_of(kind, q_lengths[i], r_lengths[i], bands ? bands[i] : band);
        // part k starts after the pair that brings the sum to k/parts of the total
        while (k < n_parts && acc >= total * (double)k / (double)n_parts)
            bounds[k++] = i + 1;
    }
    while (k <= n_parts)
        bounds[k++] = n;
    return GB2_OK;
}

}  // extern "C"

namespace {

// Runs run(ctx, first pair, pairs) for each context on its own host thread
// over the slices of the partition; returns the first failure.
template <typename Run>
int over_slices(gb2_ctx *const *ctxs, int n_ctx, const int64_t *q_lengths,
                const int64_t *r_lengths, const int32_t *bands, int32_t band, int kind, int64_t n,
                Run run)
{
    if (!ctxs || n_ctx < 1 || n < 0)
        return GB2_EINVAL;
    for (int k = 0; k < n_ctx; ++k)
        if (!ctxs[k])
            return GB2_EINVAL;
    if (n == 0)
        return GB2_OK;
    std::vector<int64_t> b(n_ctx + 1);
    int rc = gb2_partition_pairs(q_lengths, r_lengths, bands, band, kind, n, n_ctx, b.data());
    if (rc)
        return rc;
    std::vector<int> rcs(n_ctx, GB2_OK);
    std::vector<std::thread> th;
    for (int k = 0; k < n_ctx; ++k) {
        if (b[k + 1] > b[k])
            th.emplace_back([&, k] { rcs[k] = run(ctxs[k], b[k], b[k + 1] - b[k]); });
    }
    for (auto &t : th)
        t.join();
    for (int k = 0; k < n_ctx; ++k)
        if (rcs[k] != GB2_OK)
            return rcs[k];
    return GB2_OK;
}

}  // namespace

extern "C" {

int gb2_sw_banded_multi(gb2_ctx *const *ctxs, int n_ctx, const uint64_t *q_packed,
                        const int64_t *q_offsets, const int64_t *q_lengths,
                        const uint64_t *r_packed, const int64_t *r_offsets,
                        const int64_t *r_lengths, const gb2_sw_cfg *cfg, const int32_t *bands,
                        int64_t n_pairs, gb2_sw_result *out, int flags)
{
    if (!cfg || (n_pairs > 0 && (!q_offsets || !r_offsets || !out)))
        return GB2_EINVAL;
    return over_slices(ctxs, n_ctx, q_lengths, r_lengths, bands, cfg->band_width, 0, n_pairs,
                       [&](gb2_ctx *c, int64_t i0, int64_t m) {
                           return gb2_sw_banded_host(c, q_packed, q_offsets + i0, q_lengths + i0,
                                                     r_packed, r_offsets + i0, r_lengths + i0,
                                                     cfg, bands ? bands + i0 : nullptr, m,
                                                     out + i0, flags);
                       });
}

int gb2_wfa_affine_multi(gb2_ctx *const *ctxs, int n_ctx, const uint64_t *q_packed,
                         const int64_t *q_offsets, const int64_t *q_lengths,
                         const uint64_t *r_packed, const int64_t *r_offsets,
                         const int64_t *r_lengths, const gb2_wfa_cfg *cfg, int64_t n_pairs,
                         int32_t *out_cost, int flags)
{
    if (!cfg || (n_pairs > 0 && (!q_offsets || !r_offsets || !out_cost)))
        return GB2_EINVAL;
    return over_slices(ctxs, n_ctx, q_lengths, r_lengths, nullptr, 0, 1, n_pairs,
                       [&](gb2_ctx *c, int64_t i0, int64_t m) {
                           return gb2_wfa_affine_host(c, q_packed, q_offsets + i0, q_lengths + i0,
                                                      r_packed, r_offsets + i0, r_lengths + i0,
                                                      cfg, m, out_cost + i0, flags);
                       });
}

}  // extern "C"
