// api.cu -- the C ABI of libgenomics_b200.so (include/genomics_b200.h).
//
// Host runtime around the kernels: contexts (one compute stream, one copy
// stream, auxiliary streams for concurrent band classes), device-resident
// SequenceBatches uploaded through pinned staging, device-side length
// bucketing of pair lists, the chunked host-to-device pipeline of the
// end-to-end entry points, and the per-pair drop-in calls.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gb2_internal.cuh"

using namespace gb2;

#define GB2_VERSION_NUM 100  // 0.1.0

struct gb2_batch {
    uint64_t *d_packed = nullptr;
    uint64_t *d_nmask = nullptr;
    int64_t *d_offsets = nullptr;
    int64_t *d_lengths = nullptr;
    int64_t count = 0, n_words = 0, max_len = 0;
    gb2_ctx *owner = nullptr;
};

namespace {

constexpr int kAux = 4;            // auxiliary streams for concurrent band classes
constexpr int kSwClasses = 5;      // 16, 32, 64, 128, literal
constexpr int kLenBuckets = 1024;  // length buckets per class
constexpr int64_t kPinChunk = 32ll << 20;

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// One set of device buffers of the end-to-end pipeline.
struct PipeSet {
    DevBuf qw, rw, qo, ql, ro, rl, bands, out;
    cudaEvent_t copied = nullptr, done = nullptr;
};

}  // namespace

struct gb2_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t st = nullptr, st_copy = nullptr;
    cudaStream_t aux[kAux] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kAux] = {};
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::mutex mu;
    std::string last_error;
    // planning buffers
    DevBuf keys, queue, counts, seg, counters, out_sw, out_wfa, bands, scratch64, scratch32,
        work, errflag, flush, one_pair;
    // pinned staging (two halves for double buffering)
    void *pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
    void *pin_out = nullptr;
    size_t pin_out_cap = 0;
    PipeSet pipe[2];
    // stats
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_pending;
    double kernel_ms = 0.0;
    int64_t launches = 0;
    int64_t work_units = 0;
};

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
static int set_err(gb2_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->last_error = buf;
    }
    return code;
}

#define CU(ctx, call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return set_err((ctx), e_ == cudaErrorMemoryAllocation ? GB2_ENOMEM : GB2_ECUDA, \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,    \
                           __LINE__);                                                    \
    } while (0)

static int ensure(gb2_ctx *c, DevBuf &b, size_t bytes)
{
    if (bytes <= b.cap)
        return GB2_OK;
    if (b.p) {
        CU(c, cudaStreamSynchronize(c->st));
        cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    size_t cap = std::max<size_t>(bytes, 256);
    cap = (cap + 255) & ~size_t(255);
    CU(c, cudaMalloc(&b.p, cap));
    b.cap = cap;
    return GB2_OK;
}

static bool is_pinned(const void *p)
{
    if (!p)
        return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host-to-device copy on `st`.  Pinned sources go straight to the DMA
// engine; pageable sources pass through the two pinned staging halves, the
// host memcpy of one half overlapping the DMA of the other.
static int h2d(gb2_ctx *c, void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0)
        return GB2_OK;
    if (is_pinned(src)) {
        CU(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return GB2_OK;
    }
    size_t done = 0;
    int half = 0;
    while (done < bytes) {
        size_t n = std::min<size_t>(bytes - done, (size_t)kPinChunk);
        CU(c, cudaEventSynchronize(c->pin_ev[half]));
        memcpy(c->pin[half], (const char *)src + done, n);
        CU(c, cudaMemcpyAsync((char *)dst + done, c->pin[half], n, cudaMemcpyHostToDevice, st));
        CU(c, cudaEventRecord(c->pin_ev[half], st));
        done += n;
        half ^= 1;
    }
    return GB2_OK;
}

static void harvest_profile(gb2_ctx *c)
{
    for (auto &pr : c->prof_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess)
            c->kernel_ms += ms;
        else
            cudaGetLastError();
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    c->prof_pending.clear();
}

static cudaEvent_t prof_begin(gb2_ctx *c, cudaStream_t st)
{
    if (!c->profiling)
        return nullptr;
    cudaEvent_t a;
    cudaEventCreate(&a);
    cudaEventRecord(a, st);
    return a;
}

static void prof_end(gb2_ctx *c, cudaEvent_t a, cudaStream_t st)
{
    if (!a)
        return;
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, st);
    c->prof_pending.emplace_back(a, b);
}

// ---------------------------------------------------------------------------
// device-side bucketing: pairs -> queue ordered by class, then by length
// (longest first), with per-class [start, end) segments
// ---------------------------------------------------------------------------
__global__ void k_classify_sw(int64_t n, SeqView q, SeqView r, const int32_t *bands, int32_t band,
                              int fast_ok, int32_t match_pos, int32_t *keys, int *counts)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int64_t ql = q.lengths[i], rl = r.lengths[i];
    const int32_t b = bands ? bands[i] : band;
    int cls = 4;
    if (fast_ok) {
        if (b == 16)
            cls = 0;
        else if (b == 32)
            cls = 1;
        else if (b == 64)
            cls = 2;
        else if (b == 128)
            cls = 3;
    }
    if (ql >= (1 << 21) - 1 || (int64_t)match_pos * (ql < rl ? ql : rl) >= (1ll << 22))
        cls = 4;
    int64_t lb = ql >> 5;
    if (lb > kLenBuckets - 1)
        lb = kLenBuckets - 1;
    const int key = cls * kLenBuckets + (kLenBuckets - 1 - (int)lb);
    keys[i] = key;
    atomicAdd(&counts[key], 1);
}

__global__ void k_classify_wfa(int64_t n, SeqView q, SeqView r, int32_t *keys, int *counts)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int64_t l = q.lengths[i] > r.lengths[i] ? q.lengths[i] : r.lengths[i];
    int64_t lb = l >> 4;
    if (lb > kLenBuckets - 1)
        lb = kLenBuckets - 1;
    const int key = kLenBuckets - 1 - (int)lb;
    keys[i] = key;
    atomicAdd(&counts[key], 1);
}

// Exclusive scan of counts[nb] (one block); writes cursors into counts and
// class segments seg[2*c], seg[2*c+1] for nb / per_class classes.
__global__ void k_scan(int *counts, int nb, int per_class, int64_t *seg)
{
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    int s = 0;
    for (int i = t * per; i < min(nb, (t + 1) * per); ++i)
        s += counts[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        int acc = 0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            int v = part[i];
            part[i] = acc;
            acc += v;
        }
    }
    __syncthreads();
    int acc = part[t];
    for (int i = t * per; i < min(nb, (t + 1) * per); ++i) {
        int v = counts[i];
        if (i % per_class == 0)
            seg[2 * (i / per_class)] = acc;
        counts[i] = acc;
        acc += v;
        if (i % per_class == per_class - 1)
            seg[2 * (i / per_class) + 1] = acc;
    }
}

__global__ void k_scatter(int64_t n, const int32_t *keys, int *cursor, int32_t *queue)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int pos = atomicAdd(&cursor[keys[i]], 1);
    queue[pos] = (int32_t)i;
}

// ---------------------------------------------------------------------------
// Smith-Waterman core: runs n pairs of (qv, rv) into d_out on c->st.
// ---------------------------------------------------------------------------
struct SwPlanInfo {
    bool fast_ok;
    int32_t max_band;
    bool uniform_band;  // bands == nullptr
};

static int classify_band(int32_t b)
{
    switch (b) {
    case 16: return 16;
    case 32: return 32;
    case 64: return 64;
    case 128: return 128;
    default: return 0;
    }
}

static int sw_core(gb2_ctx *c, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
                   const gb2_sw_cfg *cfg, const int32_t *d_bands, const SwPlanInfo &pi, int64_t n,
                   gb2_sw_result *d_out, int flags)
{
    if (n <= 0)
        return GB2_OK;
    SwParams p{cfg->match_score, cfg->mismatch, cfg->gap_open, cfg->gap_extend};
    const int32_t match_pos = std::max(cfg->match_score, 0);
    const bool lengths_ok =
        qmax < (1 << 21) - 1 && (int64_t)match_pos * std::min(qmax, rmax) < (1ll << 22);
    const bool force_literal = (flags & GB2_FLAG_GENERIC) != 0;
    const bool batched = (flags & GB2_FLAG_BATCHED) != 0;
    const int variant = (flags >> 8) & 0xff;  // tuning knob (G/K choice), 0 = default

    // literal-kernel scratch (int64 rows), sized for the widest band
    const int64_t lit_stride = 3 * (2 * (int64_t)std::max(pi.max_band, 0) + 1);
    const int lit_grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)c->sm_count * 2);
    auto ensure_lit = [&]() -> int {
        return ensure(c, c->scratch64, (size_t)lit_grid * 128 * lit_stride * sizeof(int64_t));
    };

    // One band for every pair, pairs in input order: no planning kernels.
    if (pi.uniform_band && !batched) {
        const int cls = (pi.fast_ok && lengths_ok && !force_literal)
                            ? classify_band(cfg->band_width)
                            : 0;
        PairList pl{nullptr, n, nullptr, nullptr};
        cudaEvent_t e0 = prof_begin(c, c->st);
        if (cls > 0) {
            CU(c, launch_sw(cls, variant, qv, rv, p, cfg->band_width, nullptr, pl, d_out, nullptr,
                            0, 0, c->st));
        } else {
            int rc = ensure_lit();
            if (rc)
                return rc;
            CU(c, launch_sw(0, 0, qv, rv, p, cfg->band_width, nullptr, pl, d_out,
                            (int64_t *)c->scratch64.p, lit_stride, lit_grid, c->st));
        }
        prof_end(c, e0, c->st);
        c->launches += 1;
        return GB2_OK;
    }

    // Device planning: classify + count, scan, scatter.
    const int nb = kSwClasses * kLenBuckets;
    int rc;
    if ((rc = ensure(c, c->keys, (size_t)n * 4)) || (rc = ensure(c, c->queue, (size_t)n * 4)) ||
        (rc = ensure(c, c->counts, (size_t)nb * 4)) ||
        (rc = ensure(c, c->seg, (size_t)kSwClasses * 2 * 8)) ||
        (rc = ensure(c, c->counters, 64 * 4)))
        return rc;
    CU(c, cudaMemsetAsync(c->counts.p, 0, (size_t)nb * 4, c->st));
    CU(c, cudaMemsetAsync(c->counters.p, 0, 64 * 4, c->st));
    const int fast = (pi.fast_ok && !force_literal) ? 1 : 0;
    const int blocks = (int)((n + 255) / 256);
    k_classify_sw<<<blocks, 256, 0, c->st>>>(n, qv, rv, d_bands, cfg->band_width, fast, match_pos,
                                              (int32_t *)c->keys.p, (int *)c->counts.p);
    k_scan<<<1, 1024, 0, c->st>>>((int *)c->counts.p, nb, kLenBuckets, (int64_t *)c->seg.p);
    k_scatter<<<blocks, 256, 0, c->st>>>(n, (const int32_t *)c->keys.p, (int *)c->counts.p,
                                          (int32_t *)c->queue.p);
    CU(c, cudaGetLastError());
    c->launches += 3;

    // One persistent launch per class that can hold pairs; classes run
    // concurrently on the auxiliary streams.
    static const int cls_band[kSwClasses] = {16, 32, 64, 128, 0};
    bool need[kSwClasses] = {false, false, false, false, true};
    if (pi.uniform_band) {
        const int cb = classify_band(cfg->band_width);
        for (int k = 0; k < 4; ++k)
            need[k] = fast && cls_band[k] == cb;
        // every pair lands in the register class when band, config and the
        // batch's longest sequences all qualify: skip the literal launch
        need[4] = !(fast && cb > 0 && lengths_ok);
    } else {
        for (int k = 0; k < 4; ++k)
            need[k] = fast && cls_band[k] <= std::max<int32_t>(pi.max_band, 0);
    }
    if (need[4] && (rc = ensure_lit()))
        return rc;
    CU(c, cudaEventRecord(c->ev_fork, c->st));
    int used = 0;
    cudaEvent_t e0 = prof_begin(c, c->st);
    for (int k = 0; k < kSwClasses; ++k) {
        if (!need[k])
            continue;
        cudaStream_t s = c->aux[used % kAux];
        CU(c, cudaStreamWaitEvent(s, c->ev_fork, 0));
        PairList pl{(const int32_t *)c->queue.p, 0, (const int64_t *)c->seg.p + 2 * k,
                    (int *)c->counters.p + 16 * k};
        if (k < 4) {
            const int grid = c->sm_count * sw_blocks_per_sm(cls_band[k], variant);
            CU(c, launch_sw(cls_band[k], variant, qv, rv, p, cfg->band_width, d_bands, pl, d_out,
                            nullptr, 0, grid, s));
        } else {
            CU(c, launch_sw(0, 0, qv, rv, p, cfg->band_width, d_bands, pl, d_out,
                            (int64_t *)c->scratch64.p, lit_stride, lit_grid, s));
        }
        CU(c, cudaEventRecord(c->ev_join[used % kAux], s));
        ++used;
        c->launches += 1;
    }
    for (int i = 0; i < std::min(used, kAux); ++i)
        CU(c, cudaStreamWaitEvent(c->st, c->ev_join[i], 0));
    prof_end(c, e0, c->st);
    return GB2_OK;
}

// Validates an SW config and host band array; fills plan info.
static int sw_validate(gb2_ctx *c, const gb2_sw_cfg *cfg, const int32_t *bands, int64_t n,
                       int64_t qmax, int64_t rmax, SwPlanInfo &pi)
{
    if (!cfg)
        return set_err(c, GB2_EINVAL, "cfg is NULL");
    if (n < 0)
        return set_err(c, GB2_EINVAL, "n_pairs < 0");
    int32_t maxb = cfg->band_width;
    if (bands) {
        maxb = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (bands[i] < 0)
                return set_err(c, GB2_EINVAL, "band of pair %lld is negative", (long long)i);
            maxb = std::max(maxb, bands[i]);
        }
    } else if (cfg->band_width < 0) {
        return set_err(c, GB2_EINVAL, "band_width < 0");
    }
    const int64_t pmax = std::abs((int64_t)cfg->match_score) + std::abs((int64_t)cfg->mismatch) +
                         std::abs((int64_t)cfg->gap_open) + std::abs((int64_t)cfg->gap_extend);
    if (pmax * (qmax + rmax + 2) >= (1ll << 30) || qmax >= (1ll << 30) || rmax >= (1ll << 30))
        return set_err(c, GB2_ERANGE,
                       "scores could leave the int32 range (|params| sum %lld, lengths %lld/%lld)",
                       (long long)pmax, (long long)qmax, (long long)rmax);
    pi.fast_ok = cfg->gap_extend <= 0 && cfg->gap_open + cfg->gap_extend <= 0 && cfg->mismatch <= 0;
    pi.max_band = maxb;
    pi.uniform_band = bands == nullptr;
    return GB2_OK;
}

static SeqView view_of(const gb2_batch *b)
{
    return SeqView{b->d_packed, b->d_offsets, b->d_lengths, 0, std::max<int64_t>(b->n_words, 1)};
}

static int sync_and_check(gb2_ctx *c)
{
    CU(c, cudaStreamSynchronize(c->st));
    harvest_profile(c);
    return GB2_OK;
}

// Pinned host staging for results.
static int pin_out(gb2_ctx *c, size_t bytes)
{
    if (bytes <= c->pin_out_cap)
        return GB2_OK;
    if (c->pin_out)
        cudaFreeHost(c->pin_out);
    c->pin_out = nullptr;
    c->pin_out_cap = 0;
    CU(c, cudaMallocHost(&c->pin_out, bytes));
    c->pin_out_cap = bytes;
    return GB2_OK;
}

static int d2h_results(gb2_ctx *c, void *host, const void *dev, size_t bytes)
{
    if (bytes == 0)
        return GB2_OK;
    if (is_pinned(host)) {
        CU(c, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->st));
        return sync_and_check(c);
    }
    int rc = pin_out(c, bytes);
    if (rc)
        return rc;
    CU(c, cudaMemcpyAsync(c->pin_out, dev, bytes, cudaMemcpyDeviceToHost, c->st));
    rc = sync_and_check(c);
    if (rc)
        return rc;
    memcpy(host, c->pin_out, bytes);
    return GB2_OK;
}

// ---------------------------------------------------------------------------
// WFA core
// ---------------------------------------------------------------------------
static int gcd_h(int a, int b)
{
    while (b) {
        int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

static int wfa_validate(gb2_ctx *c, const gb2_wfa_cfg *cfg, int64_t n)
{
    if (!cfg)
        return set_err(c, GB2_EINVAL, "cfg is NULL");
    if (n < 0)
        return set_err(c, GB2_EINVAL, "n_pairs < 0");
    if (cfg->x < 1 || cfg->e < 1 || cfg->o < 0 || cfg->max_error < 0)
        return set_err(c, GB2_EINVAL, "WFA needs x >= 1, e >= 1, o >= 0, max_error >= 0");
    const int g = gcd_h(cfg->x, gcd_h(cfg->o, cfg->e));
    const int hm = std::max(cfg->x / g, (cfg->o + cfg->e) / g) + 1, hie = cfg->e / g + 1;
    if (hm > 32 || hie > 32)
        return set_err(c, GB2_EINVAL,
                       "WFA penalty ratios too large (max(x, o+e)/gcd and e/gcd must be <= 31)");
    return GB2_OK;
}

static int wfa_core(gb2_ctx *c, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
                    const gb2_wfa_cfg *cfg, int64_t n, int32_t *d_out, int flags)
{
    if (n <= 0)
        return GB2_OK;
    if (qmax >= (1ll << 30) || rmax >= (1ll << 30))
        return set_err(c, GB2_ERANGE, "sequence longer than 2^30");
    WfaParams p{cfg->x, cfg->o, cfg->e, cfg->max_error};
    const int g = gcd_h(cfg->x, gcd_h(cfg->o, cfg->e));
    const int hm = std::max(cfg->x / g, (cfg->o + cfg->e) / g) + 1, hie = cfg->e / g + 1;
    const int nslot = hm + 2 * hie;
    const int64_t slot_width = ((qmax + rmax + 5) + 31) & ~int64_t(31);
    const int blocks_per_sm = 4;
    int grid = c->sm_count * blocks_per_sm;
    const int64_t warps_needed = n;
    if ((int64_t)grid * 4 > warps_needed)
        grid = (int)std::max<int64_t>(1, (warps_needed + 3) / 4);
    const int64_t warps = (int64_t)grid * 4;
    int rc;
    if ((rc = ensure(c, c->scratch32, (size_t)warps * nslot * slot_width * 4)) ||
        (rc = ensure(c, c->errflag, 64)) || (rc = ensure(c, c->work, 64)) ||
        (rc = ensure(c, c->counters, 64 * 4)))
        return rc;
    CU(c, cudaMemsetAsync(c->errflag.p, 0, 64, c->st));
    CU(c, cudaMemsetAsync(c->work.p, 0, 64, c->st));
    CU(c, cudaMemsetAsync(c->counters.p, 0, 64 * 4, c->st));
    PairList pl{nullptr, n, nullptr, (int *)c->counters.p};
    if (flags & GB2_FLAG_BATCHED) {
        const int nb = kLenBuckets;
        if ((rc = ensure(c, c->keys, (size_t)n * 4)) || (rc = ensure(c, c->queue, (size_t)n * 4)) ||
            (rc = ensure(c, c->counts, (size_t)nb * 4)) || (rc = ensure(c, c->seg, 2 * 8)))
            return rc;
        CU(c, cudaMemsetAsync(c->counts.p, 0, (size_t)nb * 4, c->st));
        const int blocks = (int)((n + 255) / 256);
        k_classify_wfa<<<blocks, 256, 0, c->st>>>(n, qv, rv, (int32_t *)c->keys.p,
                                                   (int *)c->counts.p);
        k_scan<<<1, 1024, 0, c->st>>>((int *)c->counts.p, nb, nb, (int64_t *)c->seg.p);
        k_scatter<<<blocks, 256, 0, c->st>>>(n, (const int32_t *)c->keys.p, (int *)c->counts.p,
                                              (int32_t *)c->queue.p);
        CU(c, cudaGetLastError());
        c->launches += 3;
        pl = PairList{(const int32_t *)c->queue.p, 0, (const int64_t *)c->seg.p,
                      (int *)c->counters.p};
    }
    cudaEvent_t e0 = prof_begin(c, c->st);
    CU(c, launch_wfa(0, qv, rv, p, pl, d_out, (int32_t *)c->scratch32.p, slot_width, grid,
                     (int *)c->errflag.p, (int64_t *)c->work.p, c->st));
    prof_end(c, e0, c->st);
    c->launches += 1;
    return GB2_OK;
}

static int wfa_finish(gb2_ctx *c)
{
    int flag = 0;
    int64_t work = 0;
    CU(c, cudaMemcpyAsync(&flag, c->errflag.p, 4, cudaMemcpyDeviceToHost, c->st));
    CU(c, cudaMemcpyAsync(&work, c->work.p, 8, cudaMemcpyDeviceToHost, c->st));
    int rc = sync_and_check(c);
    if (rc)
        return rc;
    c->work_units += work;
    if (flag)
        return set_err(c, GB2_EKERNEL, "WFA kernel reported scratch overflow");
    return GB2_OK;
}

// ---------------------------------------------------------------------------
// chunked end-to-end pipeline over host SequenceBatch arrays
// ---------------------------------------------------------------------------
struct HostSide {
    const uint64_t *packed;
    const int64_t *offsets;
    const int64_t *lengths;
};

static int64_t words_for(int64_t len) { return (len + 31) / 32; }

// Word range [w0, w1) covering pairs [p0, p1) when offsets are monotone.
static void word_range(const HostSide &h, int64_t p0, int64_t p1, int64_t &w0, int64_t &w1)
{
    w0 = h.offsets[p0];
    w1 = h.offsets[p1 - 1] + words_for(h.lengths[p1 - 1]);
    if (w1 < w0)
        w1 = w0;
}

// True when sequences [0, n) follow add_sequence's append layout
// (genomics/core/sequence.mojo:44-66): each starts at or after the end of
// the previous one, so any run of pairs maps to one contiguous word range.
static bool monotone(const HostSide &h, int64_t n, int64_t &maxlen, int64_t &maxword)
{
    bool ok = true;
    int64_t prev_end = 0;
    maxlen = 0;
    maxword = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t o = h.offsets[i], l = h.lengths[i];
        const int64_t e = o + words_for(l);
        maxlen = std::max(maxlen, l);
        maxword = std::max(maxword, e);
        if (o < prev_end)
            ok = false;
        prev_end = e;
    }
    return ok;
}

template <typename RunChunk>
static int pipeline(gb2_ctx *c, const HostSide &hq, const HostSide &hr, const int32_t *bands,
                    int64_t n, size_t out_elem, void *out_host, int64_t chunk_pairs,
                    RunChunk run_chunk)
{
    int64_t qmaxlen, rmaxlen, qmaxw, rmaxw;
    const bool mq = monotone(hq, n, qmaxlen, qmaxw);
    const bool mr = monotone(hr, n, rmaxlen, rmaxw);
    for (int64_t i = 0; i < n; ++i)
        if (hq.lengths[i] < 0 || hr.lengths[i] < 0 || hq.offsets[i] < 0 || hr.offsets[i] < 0)
            return set_err(c, GB2_EINVAL, "negative offset or length at pair %lld", (long long)i);
    if (!(mq && mr))
        chunk_pairs = n;  // one chunk holding every word the pairs touch
    const int64_t nchunks = (n + chunk_pairs - 1) / chunk_pairs;
    int rc = GB2_OK;
    const bool out_pinned = is_pinned(out_host);
    if (!out_pinned && (rc = pin_out(c, (size_t)n * out_elem)))
        return rc;
    for (int64_t ci = 0; ci < nchunks; ++ci) {
        PipeSet &ps = c->pipe[ci & 1];
        const int64_t p0 = ci * chunk_pairs, p1 = std::min(n, p0 + chunk_pairs);
        const int64_t m = p1 - p0;
        int64_t qw0, qw1, rw0, rw1;
        if (mq && mr) {
            word_range(hq, p0, p1, qw0, qw1);
            word_range(hr, p0, p1, rw0, rw1);
        } else {
            qw0 = 0;
            qw1 = qmaxw;
            rw0 = 0;
            rw1 = rmaxw;
        }
        const int64_t qn = std::max<int64_t>(qw1 - qw0, 1), rn = std::max<int64_t>(rw1 - rw0, 1);
        // this buffer set's previous chunk must have finished computing
        CU(c, cudaEventSynchronize(ps.done));
        if ((rc = ensure(c, ps.qw, qn * 8)) || (rc = ensure(c, ps.rw, rn * 8)) ||
            (rc = ensure(c, ps.qo, m * 8)) || (rc = ensure(c, ps.ql, m * 8)) ||
            (rc = ensure(c, ps.ro, m * 8)) || (rc = ensure(c, ps.rl, m * 8)) ||
            (rc = ensure(c, ps.out, m * out_elem)) || (bands && (rc = ensure(c, ps.bands, m * 4))))
            return rc;
        if ((rc = h2d(c, ps.qw.p, hq.packed + qw0, (size_t)(qw1 - qw0) * 8, c->st_copy)) ||
            (rc = h2d(c, ps.rw.p, hr.packed + rw0, (size_t)(rw1 - rw0) * 8, c->st_copy)) ||
            (rc = h2d(c, ps.qo.p, hq.offsets + p0, (size_t)m * 8, c->st_copy)) ||
            (rc = h2d(c, ps.ql.p, hq.lengths + p0, (size_t)m * 8, c->st_copy)) ||
            (rc = h2d(c, ps.ro.p, hr.offsets + p0, (size_t)m * 8, c->st_copy)) ||
            (rc = h2d(c, ps.rl.p, hr.lengths + p0, (size_t)m * 8, c->st_copy)) ||
            (bands && (rc = h2d(c, ps.bands.p, bands + p0, (size_t)m * 4, c->st_copy))))
            return rc;
        CU(c, cudaEventRecord(ps.copied, c->st_copy));
        CU(c, cudaStreamWaitEvent(c->st, ps.copied, 0));
        SeqView qv{(const uint64_t *)ps.qw.p, (const int64_t *)ps.qo.p,
                   (const int64_t *)ps.ql.p, qw0, qn};
        SeqView rv{(const uint64_t *)ps.rw.p, (const int64_t *)ps.ro.p,
                   (const int64_t *)ps.rl.p, rw0, rn};
        if ((rc = run_chunk(qv, rv, qmaxlen, rmaxlen, bands ? (const int32_t *)ps.bands.p : nullptr,
                            m, ps.out.p)))
            return rc;
        void *dst = out_pinned ? (char *)out_host + p0 * out_elem
                               : (char *)c->pin_out + p0 * out_elem;
        CU(c, cudaMemcpyAsync(dst, ps.out.p, (size_t)m * out_elem, cudaMemcpyDeviceToHost, c->st));
        CU(c, cudaEventRecord(ps.done, c->st));
    }
    if ((rc = sync_and_check(c)))
        return rc;
    if (!out_pinned)
        memcpy(out_host, c->pin_out, (size_t)n * out_elem);
    return GB2_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int gb2_version(void) { return GB2_VERSION_NUM; }

const char *gb2_strerror(int status)
{
    switch (status) {
    case GB2_OK: return "ok";
    case GB2_EINVAL: return "invalid argument";
    case GB2_ENOMEM: return "out of memory";
    case GB2_ECUDA: return "CUDA runtime error";
    case GB2_ENODEV: return "no sm_100 CUDA device";
    case GB2_ERANGE: return "input outside the exact integer range";
    case GB2_ETIMEOUT: return "timed out";
    case GB2_ESTATE: return "wrong state";
    case GB2_EKERNEL: return "kernel reported an error";
    case GB2_ESCRATCH: return "request exceeds the fixed no-allocation scratch";
    default: return "unknown status";
    }
}

int gb2_create(int device, gb2_ctx **out)
{
    if (!out)
        return GB2_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GB2_ENODEV;
    }
    if (device < 0 || device >= ndev)
        return GB2_EINVAL;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return GB2_ECUDA;
    if (prop.major != 10)
        return GB2_ENODEV;
    if (cudaSetDevice(device) != cudaSuccess)
        return GB2_ECUDA;
    gb2_ctx *c = new gb2_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    bool ok = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&c->t0) == cudaSuccess && cudaEventCreate(&c->t1) == cudaSuccess;
    for (int i = 0; ok && i < kAux; ++i)
        ok = cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < 2; ++i) {
        ok = cudaMallocHost(&c->pin[i], (size_t)kPinChunk) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->pin_ev[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->pipe[i].copied, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->pipe[i].done, cudaEventDisableTiming) == cudaSuccess;
        if (ok) {
            cudaEventRecord(c->pin_ev[i], c->st);
            cudaEventRecord(c->pipe[i].done, c->st);
        }
    }
    if (!ok) {
        cudaGetLastError();
        gb2_destroy(c);
        return GB2_ECUDA;
    }
    *out = c;
    return GB2_OK;
}

int gb2_destroy(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    cudaSetDevice(c->device);
    if (c->st)
        cudaStreamSynchronize(c->st);
    if (c->st_copy)
        cudaStreamSynchronize(c->st_copy);
    harvest_profile(c);
    DevBuf *bufs[] = {&c->keys,      &c->queue,     &c->counts, &c->seg,   &c->counters,
                      &c->out_sw,    &c->out_wfa,   &c->bands,  &c->scratch64,
                      &c->scratch32, &c->work,      &c->errflag, &c->flush, &c->one_pair};
    for (DevBuf *b : bufs)
        if (b->p)
            cudaFree(b->p);
    for (int i = 0; i < 2; ++i) {
        PipeSet &ps = c->pipe[i];
        DevBuf *pb[] = {&ps.qw, &ps.rw, &ps.qo, &ps.ql, &ps.ro, &ps.rl, &ps.bands, &ps.out};
        for (DevBuf *b : pb)
            if (b->p)
                cudaFree(b->p);
        if (ps.copied)
            cudaEventDestroy(ps.copied);
        if (ps.done)
            cudaEventDestroy(ps.done);
        if (c->pin[i])
            cudaFreeHost(c->pin[i]);
        if (c->pin_ev[i])
            cudaEventDestroy(c->pin_ev[i]);
    }
    if (c->pin_out)
        cudaFreeHost(c->pin_out);
    for (int i = 0; i < kAux; ++i) {
        if (c->aux[i])
            cudaStreamDestroy(c->aux[i]);
        if (c->ev_join[i])
            cudaEventDestroy(c->ev_join[i]);
    }
    if (c->ev_fork)
        cudaEventDestroy(c->ev_fork);
    if (c->t0)
        cudaEventDestroy(c->t0);
    if (c->t1)
        cudaEventDestroy(c->t1);
    if (c->st)
        cudaStreamDestroy(c->st);
    if (c->st_copy)
        cudaStreamDestroy(c->st_copy);
    delete c;
    return GB2_OK;
}

int gb2_sync(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    CU(c, cudaStreamSynchronize(c->st_copy));
    return sync_and_check(c);
}

const char *gb2_last_error(gb2_ctx *c) { return c ? c->last_error.c_str() : "no context"; }

int gb2_batch_upload(gb2_ctx *c, const uint64_t *packed, int64_t n_words, const uint64_t *nmask,
                     const int64_t *offsets, const int64_t *lengths, int64_t count,
                     gb2_batch **out)
{
    if (!c || !out)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    *out = nullptr;
    if (count < 0 || n_words < 0 || (count > 0 && (!offsets || !lengths)) ||
        (n_words > 0 && !packed))
        return set_err(c, GB2_EINVAL, "batch arrays missing or sizes negative");
    int64_t maxlen = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (lengths[i] < 0 || offsets[i] < 0 || offsets[i] + words_for(lengths[i]) > n_words)
            return set_err(c, GB2_EINVAL, "sequence %lld lies outside the packed words",
                           (long long)i);
        maxlen = std::max(maxlen, lengths[i]);
    }
    gb2_batch *b = new gb2_batch();
    b->owner = c;
    b->count = count;
    b->n_words = n_words;
    b->max_len = maxlen;
    const size_t wb = (size_t)std::max<int64_t>(n_words, 1) * 8;
    const size_t sb = (size_t)std::max<int64_t>(count, 1) * 8;
    cudaError_t e = cudaMalloc(&b->d_packed, wb);
    if (e == cudaSuccess && nmask)
        e = cudaMalloc(&b->d_nmask, wb);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_offsets, sb);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_lengths, sb);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(b->d_packed);
        cudaFree(b->d_nmask);
        cudaFree(b->d_offsets);
        cudaFree(b->d_lengths);
        delete b;
        return set_err(c, GB2_ENOMEM, "device allocation of a %lld-word batch failed",
                       (long long)n_words);
    }
    int rc = GB2_OK;
    if (n_words == 0)
        cudaMemsetAsync(b->d_packed, 0, 8, c->st);
    if (!rc)
        rc = h2d(c, b->d_packed, packed, (size_t)n_words * 8, c->st);
    if (!rc && nmask)
        rc = h2d(c, b->d_nmask, nmask, (size_t)n_words * 8, c->st);
    if (!rc)
        rc = h2d(c, b->d_offsets, offsets, (size_t)count * 8, c->st);
    if (!rc)
        rc = h2d(c, b->d_lengths, lengths, (size_t)count * 8, c->st);
    if (!rc)
        rc = sync_and_check(c);
    if (rc) {
        cudaFree(b->d_packed);
        cudaFree(b->d_nmask);
        cudaFree(b->d_offsets);
        cudaFree(b->d_lengths);
        delete b;
        return rc;
    }
    *out = b;
    return GB2_OK;
}

int gb2_batch_free(gb2_ctx *c, gb2_batch *b)
{
    if (!c || !b || b->owner != c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->st);
    cudaFree(b->d_packed);
    cudaFree(b->d_nmask);
    cudaFree(b->d_offsets);
    cudaFree(b->d_lengths);
    delete b;
    return GB2_OK;
}

int gb2_batch_info(const gb2_batch *b, int64_t *count, int64_t *n_words)
{
    if (!b)
        return GB2_EINVAL;
    if (count)
        *count = b->count;
    if (n_words)
        *n_words = b->n_words;
    return GB2_OK;
}

int gb2_sw_banded(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_sw_cfg *cfg,
                  const int32_t *bands, int64_t n, gb2_sw_result *out, int flags)
{
    if (!c || !q || !r)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (q->owner != c || r->owner != c)
        return set_err(c, GB2_EINVAL, "batch belongs to another context");
    if (n > q->count || n > r->count)
        return set_err(c, GB2_EINVAL, "n_pairs exceeds a batch's sequence count");
    if (n > 0 && !out)
        return set_err(c, GB2_EINVAL, "out is NULL");
    SwPlanInfo pi;
    int rc = sw_validate(c, cfg, bands, n, q->max_len, r->max_len, pi);
    if (rc)
        return rc;
    if (n == 0)
        return GB2_OK;
    if ((rc = ensure(c, c->out_sw, (size_t)n * sizeof(gb2_sw_result))))
        return rc;
    const int32_t *d_bands = nullptr;
    if (bands) {
        if ((rc = ensure(c, c->bands, (size_t)n * 4)) ||
            (rc = h2d(c, c->bands.p, bands, (size_t)n * 4, c->st)))
            return rc;
        d_bands = (const int32_t *)c->bands.p;
    }
    if ((rc = sw_core(c, view_of(q), view_of(r), q->max_len, r->max_len, cfg, d_bands, pi, n,
                      (gb2_sw_result *)c->out_sw.p, flags)))
        return rc;
    return d2h_results(c, out, c->out_sw.p, (size_t)n * sizeof(gb2_sw_result));
}

int gb2_sw_banded_host(gb2_ctx *c, const uint64_t *q_packed, const int64_t *q_offsets,
                       const int64_t *q_lengths, const uint64_t *r_packed,
                       const int64_t *r_offsets, const int64_t *r_lengths, const gb2_sw_cfg *cfg,
                       const int32_t *bands, int64_t n, gb2_sw_result *out, int flags)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (n > 0 && (!q_packed || !q_offsets || !q_lengths || !r_packed || !r_offsets ||
                  !r_lengths || !out))
        return set_err(c, GB2_EINVAL, "NULL array");
    int64_t qmax = 0, rmax = 0;
    for (int64_t i = 0; i < n; ++i) {
        qmax = std::max(qmax, q_lengths[i]);
        rmax = std::max(rmax, r_lengths[i]);
    }
    SwPlanInfo pi;
    int rc = sw_validate(c, cfg, bands, n, qmax, rmax, pi);
    if (rc || n == 0)
        return rc;
    HostSide hq{q_packed, q_offsets, q_lengths}, hr{r_packed, r_offsets, r_lengths};
    const int64_t chunk = std::max<int64_t>(4096, (n + 7) / 8);
    return pipeline(c, hq, hr, bands, n, sizeof(gb2_sw_result), out, chunk,
                    [&](SeqView qv, SeqView rv, int64_t qm, int64_t rm, const int32_t *db,
                        int64_t m, void *dout) {
                        return sw_core(c, qv, rv, qm, rm, cfg, db, pi, m, (gb2_sw_result *)dout,
                                       flags);
                    });
}

int gb2_sw_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                int64_t rlen, const gb2_sw_cfg *cfg, gb2_sw_result *out)
{
    if (!c)
        return GB2_EINVAL;
    if (!out || qlen < 0 || rlen < 0 || (qlen > 0 && !q_words) || (rlen > 0 && !r_words))
        return set_err(c, GB2_EINVAL, "bad pair arguments");
    int64_t qo = 0, ro = 0;
    static const uint64_t zero = 0;
    return gb2_sw_banded_host(c, qlen ? q_words : &zero, &qo, &qlen, rlen ? r_words : &zero, &ro,
                              &rlen, cfg, nullptr, 1, out, GB2_FLAG_PLAIN);
}

int gb2_wfa_affine(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_wfa_cfg *cfg,
                   int64_t n, int32_t *out, int flags)
{
    if (!c || !q || !r)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (q->owner != c || r->owner != c)
        return set_err(c, GB2_EINVAL, "batch belongs to another context");
    if (n > q->count || n > r->count)
        return set_err(c, GB2_EINVAL, "n_pairs exceeds a batch's sequence count");
    if (n > 0 && !out)
        return set_err(c, GB2_EINVAL, "out is NULL");
    int rc = wfa_validate(c, cfg, n);
    if (rc || n == 0)
        return rc;
    if ((rc = ensure(c, c->out_wfa, (size_t)n * 4)))
        return rc;
    if ((rc = wfa_core(c, view_of(q), view_of(r), q->max_len, r->max_len, cfg, n,
                       (int32_t *)c->out_wfa.p, flags)))
        return rc;
    if ((rc = wfa_finish(c)))
        return rc;
    return d2h_results(c, out, c->out_wfa.p, (size_t)n * 4);
}

int gb2_wfa_affine_host(gb2_ctx *c, const uint64_t *q_packed, const int64_t *q_offsets,
                        const int64_t *q_lengths, const uint64_t *r_packed,
                        const int64_t *r_offsets, const int64_t *r_lengths,
                        const gb2_wfa_cfg *cfg, int64_t n, int32_t *out, int flags)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (n > 0 && (!q_packed || !q_offsets || !q_lengths || !r_packed || !r_offsets ||
                  !r_lengths || !out))
        return set_err(c, GB2_EINVAL, "NULL array");
    int rc = wfa_validate(c, cfg, n);
    if (rc || n == 0)
        return rc;
    HostSide hq{q_packed, q_offsets, q_lengths}, hr{r_packed, r_offsets, r_lengths};
    const int64_t chunk = std::max<int64_t>(1024, (n + 3) / 4);
    rc = pipeline(c, hq, hr, nullptr, n, 4, out, chunk,
                  [&](SeqView qv, SeqView rv, int64_t qm, int64_t rm, const int32_t *,
                      int64_t m, void *dout) {
                      return wfa_core(c, qv, rv, qm, rm, cfg, m, (int32_t *)dout, flags);
                  });
    if (rc)
        return rc;
    return wfa_finish(c);
}

int gb2_wfa_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                 int64_t rlen, const gb2_wfa_cfg *cfg, int32_t *out)
{
    if (!c)
        return GB2_EINVAL;
    if (!out || qlen < 0 || rlen < 0 || (qlen > 0 && !q_words) || (rlen > 0 && !r_words))
        return set_err(c, GB2_EINVAL, "bad pair arguments");
    int64_t qo = 0, ro = 0;
    static const uint64_t zero = 0;
    return gb2_wfa_affine_host(c, qlen ? q_words : &zero, &qo, &qlen, rlen ? r_words : &zero, &ro,
                               &rlen, cfg, 1, out, GB2_FLAG_PLAIN);
}

int gb2_host_alloc(int64_t bytes, void **out)
{
    if (!out || bytes < 0)
        return GB2_EINVAL;
    *out = nullptr;
    if (cudaMallocHost(out, (size_t)std::max<int64_t>(bytes, 8)) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return GB2_ENOMEM;
    }
    return GB2_OK;
}

int gb2_host_free(void *p)
{
    if (!p)
        return GB2_OK;
    return cudaFreeHost(p) == cudaSuccess ? GB2_OK : GB2_ECUDA;
}

int gb2_timer_start(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    cudaSetDevice(c->device);
    CU(c, cudaEventRecord(c->t0, c->st));
    return GB2_OK;
}

int gb2_timer_stop(gb2_ctx *c, float *ms)
{
    if (!c || !ms)
        return GB2_EINVAL;
    cudaSetDevice(c->device);
    CU(c, cudaEventRecord(c->t1, c->st));
    CU(c, cudaEventSynchronize(c->t1));
    CU(c, cudaEventElapsedTime(ms, c->t0, c->t1));
    return GB2_OK;
}

int gb2_stats(gb2_ctx *c, double *kernel_ms, int64_t *launches, int64_t *work_units)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    CU(c, cudaStreamSynchronize(c->st));
    harvest_profile(c);
    if (kernel_ms)
        *kernel_ms = c->kernel_ms;
    if (launches)
        *launches = c->launches;
    if (work_units)
        *work_units = c->work_units;
    return GB2_OK;
}

int gb2_stats_reset(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    CU(c, cudaStreamSynchronize(c->st));
    harvest_profile(c);
    c->kernel_ms = 0;
    c->launches = 0;
    c->work_units = 0;
    return GB2_OK;
}

int gb2_set_profiling(gb2_ctx *c, int enable)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    c->profiling = enable != 0;
    return GB2_OK;
}

int gb2_flush_l2(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const size_t bytes = 256ull << 20;  // twice the 126 MB L2
    int rc = ensure(c, c->flush, bytes);
    if (rc)
        return rc;
    CU(c, cudaMemsetAsync(c->flush.p, c->launches & 0xff, bytes, c->st));
    return GB2_OK;
}

int gb2_int_peak(gb2_ctx *c, int kind, double *gops)
{
    if (!c || !gops || kind < 0 || kind > 7)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    int rc = ensure(c, c->work, 64);
    if (rc)
        return rc;
    CU(c, cudaMemsetAsync(c->work.p, 0, 64, c->st));
    const int block = 256, grid = c->sm_count * 8, iters = 4096;
    // warm-up, then timed
    CU(c, launch_int_peak(kind, grid, block, 64, (uint32_t *)c->work.p, c->st));
    CU(c, cudaEventRecord(c->t0, c->st));
    CU(c, launch_int_peak(kind, grid, block, iters, (uint32_t *)c->work.p, c->st));
    CU(c, cudaEventRecord(c->t1, c->st));
    CU(c, cudaEventSynchronize(c->t1));
    float ms = 0.f;
    CU(c, cudaEventElapsedTime(&ms, c->t0, c->t1));
    const double ops = (double)grid * block * iters * 8.0;
    *gops = ops / (ms * 1e-3) / 1e9;
    return GB2_OK;
}

}  // extern "C"
