// wfa_cigar.cu -- host side of gap-affine WFA with CIGAR traceback.
//
// wfa_affine_cigar_cpu (genomics/cpu/align_cpu.mojo:380-623) keeps M before
// and after extension, I and D for every score up to the optimum and every
// diagonal in [-max_err, max_err], then walks back from (opt, qlen - rlen).
// Here a first pass is the cost kernel, which also reports how many bytes
// each pair's history record will take; a second pass (wfa_cigar_kernel in
// wfa_kernels.cu) re-runs each pair's forward recurrences with the cost
// kernel's own code in history mode, appending per visited score the
// M-after-extension values and one decision byte per diagonal to the pair's
// record in an arena sized from the first pass, and walks the record back
// into CIGAR runs (wfa_trace.cuh).  The host groups pairs, largest records
// first, so the records of a group fit the arena, then gathers every pair's
// runs into the caller's array.
//
// A history record costs 4 B + 1 B per visited cell plus 12 B per score,
// against the reference's 4 int64 arrays over (max_err+1) x (2 max_err+1).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "runtime.cuh"

namespace gb2 {
namespace {

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
    const int arena_mib = (int)(((unsigned)flags >> 24) & 0xff);
    flags &= 0x00ffffff;
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
    int64_t budget = std::min<int64_t>((int64_t)free_b / 2,
                                       arena_mib ? (int64_t)arena_mib << 20 : kCigarArenaCap);
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
    int64_t grid = (int64_t)c->sm_count * wfa_cigar_blocks_per_sm();
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
        // the largest records of the group, one wave of blocks, one pair per block
        const int gg = (int)std::min<int64_t>(grid, (m + 3) / 4);
        const int64_t n_team = std::min<int64_t>(gg, m);
        GB2_CU(c, cudaMemsetAsync(x.counters.p, 0, 256, x.st));
        GB2_CU(c, launch_wfa_cigar(qv, rv, p, (const int32_t *)cb.pairs.p, m, n_team,
                                   (int *)x.counters.p, (const int32_t *)cb.cost.p,
                                   (const int64_t *)cb.hist.p,
                                   (const int64_t *)cb.arena_off.p, (uint8_t *)cb.arena.p,
                                   (int32_t *)x.scratch32.p, slot_width, gg,
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

static int gb2_wfa_cigar_impl(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_wfa_cfg *cfg,
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

int gb2_wfa_cigar(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_wfa_cfg *cfg,
                  int64_t n, int32_t *cost, uint32_t *runs, int64_t runs_cap,
                  int64_t *run_offsets, int flags)
{
    return drain_on_error(c, gb2_wfa_cigar_impl(c, q, r, cfg, n, cost, runs, runs_cap, run_offsets, flags));
}

static int gb2_wfa_cigar_pair_impl(gb2_ctx *c, const uint64_t *q_words, int64_t qlen,
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

int gb2_wfa_cigar_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen,
                       const uint64_t *r_words, int64_t rlen, const gb2_wfa_cfg *cfg,
                       int32_t *cost, char *cigar, int64_t cap)
{
    return drain_on_error(c, gb2_wfa_cigar_pair_impl(c, q_words, qlen, r_words, rlen, cfg, cost, cigar, cap));
}

}  // extern "C"
