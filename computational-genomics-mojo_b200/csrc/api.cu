// api.cu -- the C ABI of libgenomics_b200.so (include/genomics_b200.h).
//
// Host runtime around the kernels: contexts and executors (a stream plus
// the planning and scratch buffers its launches use), device-resident
// SequenceBatches uploaded through pinned staging, device-side length
// bucketing of pair lists, the chunked host-to-device pipeline of the
// end-to-end entry points, and the per-pair drop-in calls.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>

#include "runtime.cuh"

using namespace gb2;

#define GB2_VERSION_NUM 100  // 0.1.0
#define CU GB2_CU

namespace {
constexpr size_t kCounterBytes = 4096;  // dynamic-queue counters, 128 B apart
constexpr int kCounterStride = 32;      // ints between the counters of two classes
}  // namespace

namespace gb2 {

// ---------------------------------------------------------------------------
// plumbing
// ---------------------------------------------------------------------------
int set_err(gb2_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        std::lock_guard<std::mutex> lk(c->err_mu);
        c->last_error = buf;
    }
    return code;
}

std::atomic<int64_t> g_fail_dev{-1}, g_fail_pin{-1};

int drain_on_error(gb2_ctx *c, int rc)
{
    if (rc == GB2_OK || !c)
        return rc;
    cudaSetDevice(c->device);
    auto drain = [](cudaStream_t s) {
        if (s)
            cudaStreamSynchronize(s);
    };
    for (Exec *x : {&c->x, &c->x2}) {
        drain(x->st);
        for (int i = 0; i < kAux; ++i)
            drain(x->aux[i]);
    }
    drain(c->st_copy);
    drain(c->st_prep);
    drain(c->st_back);
    cudaGetLastError();
    return rc;
}

int exec_init(Exec &x)
{
    bool ok = cudaStreamCreateWithFlags(&x.st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&x.ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < kAux; ++i)
        ok = cudaStreamCreateWithFlags(&x.aux[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&x.ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok)
        cudaGetLastError();
    return ok ? GB2_OK : GB2_ECUDA;
}

void exec_free(Exec &x)
{
    if (x.st)
        cudaStreamSynchronize(x.st);
    for (int i = 0; i < kAux; ++i)
        if (x.aux[i])
            cudaStreamSynchronize(x.aux[i]);
    DevBuf *bufs[] = {&x.keys,      &x.queue,     &x.counts, &x.seg,   &x.counters,
                      &x.scratch64, &x.scratch32, &x.work,   &x.errflag, &x.tierq,
                      &x.dumps,     &x.ubound};
    for (DevBuf *b : bufs)
        if (b->p) {
            cudaFree(b->p);
            b->p = nullptr;
            b->cap = 0;
        }
    for (int i = 0; i < kAux; ++i) {
        if (x.aux[i])
            cudaStreamDestroy(x.aux[i]);
        if (x.ev_join[i])
            cudaEventDestroy(x.ev_join[i]);
        x.aux[i] = nullptr;
        x.ev_join[i] = nullptr;
    }
    if (x.ev_fork)
        cudaEventDestroy(x.ev_fork);
    if (x.st)
        cudaStreamDestroy(x.st);
    x.ev_fork = nullptr;
    x.st = nullptr;
}

int ensure(gb2_ctx *c, DevBuf &b, size_t bytes, cudaStream_t st)
{
    if (bytes <= b.cap)
        return GB2_OK;
    if (b.pool) {  // stream-ordered: the old buffer is freed after the work queued on st
        size_t cap = std::max<size_t>(bytes + bytes / 2, 256);
        cap = (cap + 255) & ~size_t(255);
        ++c->buf_gen;
        if (b.p)
            CU(c, cudaFreeAsync(b.p, st));
        b.p = nullptr;
        b.cap = 0;
        CU(c, dev_alloc_pool(&b.p, cap, b.pool, st));
        b.cap = cap;
        return GB2_OK;
    }
    if (b.p) {
        CU(c, cudaStreamSynchronize(st));
        cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    size_t cap = std::max<size_t>(bytes, 256);
    cap = (cap + 255) & ~size_t(255);
    ++c->buf_gen;  // captured graphs hold buffer addresses: they are stale now
    CU(c, dev_alloc(&b.p, cap));
    b.cap = cap;
    return GB2_OK;
}

bool is_pinned(const void *p)
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

int h2d(gb2_ctx *c, void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0)
        return GB2_OK;
    if (is_pinned(src)) {
        CU(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return GB2_OK;
    }
    std::lock_guard<std::mutex> lk(c->pin_mu);
    size_t done = 0;
    int half = 0;
    while (done < bytes) {
        const size_t n = std::min<size_t>(bytes - done, (size_t)kPinChunk);
        CU(c, cudaEventSynchronize(c->pin_ev[half]));
        memcpy(c->pin[half], (const char *)src + done, n);
        CU(c, cudaMemcpyAsync((char *)dst + done, c->pin[half], n, cudaMemcpyHostToDevice, st));
        CU(c, cudaEventRecord(c->pin_ev[half], st));
        done += n;
        half ^= 1;
    }
    return GB2_OK;
}

int64_t words_for(int64_t len) { return (len + 31) / 32; }

void harvest_profile(gb2_ctx *c)
{
    std::lock_guard<std::mutex> lk(c->prof_mu);
    for (auto &pr : c->prof_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(pr.second) == cudaSuccess &&
            cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess)
            c->kernel_ms += ms;
        else
            cudaGetLastError();
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    c->prof_pending.clear();
}

}  // namespace gb2

static cudaEvent_t prof_begin(gb2_ctx *c, cudaStream_t st)
{
    if (!c->profiling.load())
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
    std::lock_guard<std::mutex> lk(c->prof_mu);
    c->prof_pending.emplace_back(a, b);
}

// ---------------------------------------------------------------------------
// device-side bucketing: pairs -> queue ordered by class, then by length
// (longest first), with per-class [start, end) segments
// ---------------------------------------------------------------------------
// One atomic per distinct key in the warp (lanes with equal keys aggregate):
// a uniform batch would otherwise serialise every pair on one counter.
__device__ __forceinline__ void count_key(int *counts, int key)
{
    const unsigned mask = __match_any_sync(__activemask(), key);
    if ((threadIdx.x & 31) == __ffs(mask) - 1)
        atomicAdd(&counts[key], __popc(mask));
}

__global__ void k_classify_sw(int64_t n, SeqView q, SeqView r, const int32_t *bands, int32_t band,
                              int fast_ok, int pack_ok, int wide_ok, int32_t match_pos,
                              int32_t *keys, int *counts)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int64_t ql = q.lengths[i], rl = r.lengths[i];
    const int32_t b = bands ? bands[i] : band;
    // bound on every H the kernels compute (the row past the query end included)
    const int64_t hmax = (int64_t)match_pos * ((ql < rl ? ql : rl) + 1);
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
    if (ql >= (1 << 21) - 1 || hmax >= (1ll << 22))
        cls = 4;
    if (pack_ok && hmax <= kPackHmax && (cls == 0 || cls == 1))
        cls = cls == 0 ? 5 : 6;
    else if (wide_ok && hmax <= kWideHmax && cls <= 3)
        cls = 7 + cls;
    int64_t lb = ql >> 5;
    if (lb > kLenBuckets - 1)
        lb = kLenBuckets - 1;
    const int key = cls * kLenBuckets + (kLenBuckets - 1 - (int)lb);
    keys[i] = key;
    count_key(counts, key);
}

// WFA pairs are ordered longest first (length buckets of 16 bases, the
// longer of the two sequences), so the pairs with the longest dependency
// chains start first.
__global__ void k_classify_wfa(int64_t n, SeqView q, SeqView r, int32_t *keys, int *counts)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int64_t l = q.lengths[i] > r.lengths[i] ? q.lengths[i] : r.lengths[i];
    int64_t lb = l >> 4;
    if (lb > kLenBuckets - 1)
        lb = kLenBuckets - 1;
    const int key = kLenBuckets - 1 - (int)lb;
    keys[i] = key;
    count_key(counts, key);
}

// Splits the longest-first WFA queue after its scan: the first
// min(team_pairs, pairs at least team_len long) pairs are aligned by a whole
// block each, the rest by one warp each.  seg = {0, split, split, n}.
__global__ void k_split_wfa(const int *starts, int64_t n, int64_t team_len, int64_t team_pairs,
                            int64_t *seg)
{
    const int64_t lb = team_len >> 4;
    int64_t longs = lb > kLenBuckets - 1 ? 0 : starts[kLenBuckets - (int)lb];
    if (lb <= 0)
        longs = n;
    const int64_t split = longs < team_pairs ? longs : team_pairs;
    seg[0] = 0;
    seg[1] = split;
    seg[2] = split;
    seg[3] = n;
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
            const int v = part[i];
            part[i] = acc;
            acc += v;
        }
    }
    __syncthreads();
    int acc = part[t];
    for (int i = t * per; i < min(nb, (t + 1) * per); ++i) {
        const int v = counts[i];
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
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int key = keys[i];
    const unsigned mask = __match_any_sync(__activemask(), key);
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    int pos = 0;
    if (lane == leader)
        pos = atomicAdd(&cursor[key], __popc(mask));
    pos = __shfl_sync(mask, pos, leader) + __popc(mask & ((1u << lane) - 1u));
    queue[pos] = (int32_t)i;
}

// ---------------------------------------------------------------------------
// Smith-Waterman core
// ---------------------------------------------------------------------------
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

namespace gb2 {

int sw_core(gb2_ctx *c, Exec &x, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
            const gb2_sw_cfg *cfg, const int32_t *d_bands, const SwPlanInfo &pi, int64_t n,
            gb2_sw_result *d_out, int flags, bool profile)
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
    // per band class: the caller's variant, else the one installed by the tuner,
    // else for a small batch (which leaves most SMs idle) the variant with the
    // most lanes per pair, which shortens each pair's row loop; else the default
    auto var_of = [&](int cls) -> int {
        if (variant)
            return variant;
        const int slot = cls == 16 ? 0 : cls == 32 ? 1 : cls == 64 ? 2 : cls == 128 ? 3 : -1;
        if (slot < 0)
            return 0;
        if (c->tune_sw[slot])
            return c->tune_sw[slot];
        if (n <= kSwSmallBatch)
            return cls == 32 ? 2 : 1;  // G = 2, 4, 4, 8 for bands 16, 32, 64, 128
        return 0;
    };

    // literal-kernel scratch (int64 rows), sized for the widest band
    const int64_t lit_stride = 3 * (2 * (int64_t)std::max(pi.max_band, 0) + 1);
    const int lit_grid = (int)std::min<int64_t>((n + 127) / 128, (int64_t)c->sm_count * 2);
    auto ensure_lit = [&]() -> int {
        return ensure(c, x.scratch64, (size_t)lit_grid * 128 * lit_stride * sizeof(int64_t), x.st);
    };

    if ((flags & GB2_FLAG_NAIVE) && !force_literal && pi.max_band <= kSwNaiveMaxBand) {
        // the baseline the batched path is measured against: one block per pair,
        // input order, no planning, per-pair bands read by the kernel
        cudaEvent_t e0 = profile ? prof_begin(c, x.st) : nullptr;
        CU(c, launch_sw_naive(qv, rv, p, cfg->band_width, d_bands, std::max(pi.max_band, 0), n,
                              d_out, x.st));
        prof_end(c, e0, x.st);
        c->launches += 1;
        return GB2_OK;
    }
    const bool pack = pi.pack_ok && !force_literal && !(flags & GB2_FLAG_INT32);
    // Wide keys: a small batch leaves most SMs idle and its longest pair's row loop
    // is the call's critical path, which the int32 kernels with the most lanes per
    // pair (var_of) shorten; one thread per pair of the packed kernel does not (2,000
    // mixed-band pairs: 2.4 ms against 4.4; one pair per call: about 1,800 against
    // 1,100 pairs/s).  GB2_FLAG_PACKED keeps the packed kernel for small batches too.
    const bool wide =
        pack && pi.wide_ok && (n > kSwSmallBatch || (flags & GB2_FLAG_PACKED) != 0);
    const int64_t hbound = (int64_t)match_pos * (std::min(qmax, rmax) + 1);
    const bool pack_lengths = hbound <= kPackHmax;
    const bool wide_lengths = hbound <= kWideHmax;
    // One band for every pair, pairs in input order: no planning kernels.
    // The batched path takes it too when the lengths are narrow (nothing to
    // sort), with a dynamic pair counter.
    if (pi.uniform_band && (!batched || pi.narrow_lengths)) {
        int cls = (pi.fast_ok && lengths_ok && !force_literal) ? classify_band(cfg->band_width) : 0;
        if ((cls == 16 || cls == 32) && pack && pack_lengths)
            cls |= kPack16;
        else if (cls > 0 && wide && wide_lengths)
            cls |= kPackWide;
        PairList pl{nullptr, n, nullptr, nullptr};
        int grid = 0;  // one pair per thread, pairs in input order
        if (batched && cls > 0) {  // persistent blocks taking pairs from a counter
            int rc;
            if ((rc = ensure(c, x.counters, kCounterBytes, x.st)))
                return rc;
            CU(c, cudaMemsetAsync(x.counters.p, 0, 64, x.st));
            pl.counter = (int *)x.counters.p;
            grid = c->sm_count * sw_blocks_per_sm(cls, var_of(cls));
        }
        cudaEvent_t e0 = profile ? prof_begin(c, x.st) : nullptr;
        if (cls > 0) {
            CU(c, launch_sw(cls, var_of(cls), qv, rv, p, cfg->band_width, nullptr, pl, d_out, nullptr,
                            0, grid, x.st));
        } else {
            const int rc = ensure_lit();
            if (rc)
                return rc;
            CU(c, launch_sw(0, 0, qv, rv, p, cfg->band_width, nullptr, pl, d_out,
                            (int64_t *)x.scratch64.p, lit_stride, lit_grid, x.st));
        }
        prof_end(c, e0, x.st);
        c->launches += 1;
        return GB2_OK;
    }

    // Device planning: classify + count, scan, scatter.
    const int nb = kSwClasses * kLenBuckets;
    int rc;
    if ((rc = ensure(c, x.keys, (size_t)n * 4, x.st)) ||
        (rc = ensure(c, x.queue, (size_t)n * 4, x.st)) ||
        (rc = ensure(c, x.counts, (size_t)nb * 4, x.st)) ||
        (rc = ensure(c, x.seg, (size_t)kSwClasses * 2 * 8, x.st)) ||
        (rc = ensure(c, x.counters, kCounterBytes, x.st)))
        return rc;
    CU(c, cudaMemsetAsync(x.counts.p, 0, (size_t)nb * 4, x.st));
    CU(c, cudaMemsetAsync(x.counters.p, 0, kCounterBytes, x.st));
    const int fast = (pi.fast_ok && !force_literal) ? 1 : 0;
    const int blocks = (int)((n + 255) / 256);
    k_classify_sw<<<blocks, 256, 0, x.st>>>(n, qv, rv, d_bands, cfg->band_width, fast,
                                             pack ? 1 : 0, wide ? 1 : 0, match_pos,
                                             (int32_t *)x.keys.p, (int *)x.counts.p);
    k_scan<<<1, 1024, 0, x.st>>>((int *)x.counts.p, nb, kLenBuckets, (int64_t *)x.seg.p);
    k_scatter<<<blocks, 256, 0, x.st>>>(n, (const int32_t *)x.keys.p, (int *)x.counts.p,
                                         (int32_t *)x.queue.p);
    CU(c, cudaGetLastError());
    c->launches += 3;

    // One persistent launch per class that can hold pairs; classes run
    // concurrently on the auxiliary streams.
    static const int cls_band[kSwClasses] = {16, 32, 64, 128, 0, 16 | kPack16, 32 | kPack16,
                                             16 | kPackWide, 32 | kPackWide, 64 | kPackWide,
                                             128 | kPackWide};
    static_assert(kSwClasses * kCounterStride * 4 <= (int)kCounterBytes, "counter space");
    bool need[kSwClasses] = {false, false, false, false, true, false,
                             false, false, false, false, false};
    if (pi.uniform_band) {
        const int cb = classify_band(cfg->band_width);
        for (int k = 0; k < 4; ++k)
            need[k] = fast && cls_band[k] == cb;
        need[5] = pack && cb == 16;
        need[6] = pack && cb == 32;
        for (int k = 0; k < 4; ++k)
            need[7 + k] = wide && cls_band[k] == cb;
        // when the batch's longest sequences qualify, every pair lands in one
        // class: skip the launches that would find nothing
        if (need[5] || need[6]) {
            need[0] = need[0] && !pack_lengths;
            need[1] = need[1] && !pack_lengths;
            for (int k = 7; k < 9; ++k)
                need[k] = need[k] && !pack_lengths;
        }
        for (int k = 0; k < 4; ++k)
            if (need[7 + k])
                need[k] = need[k] && !wide_lengths;
        need[4] = !(fast && cb > 0 && lengths_ok);
    } else {
        for (int k = 0; k < 4; ++k)
            need[k] = fast && cls_band[k] <= std::max<int32_t>(pi.max_band, 0);
        need[5] = pack && pi.max_band >= 16;
        need[6] = pack && pi.max_band >= 32;
        for (int k = 0; k < 4; ++k)
            need[7 + k] = wide && (cls_band[k] & 0xff) <= std::max<int32_t>(pi.max_band, 0);
    }
    if (need[4] && (rc = ensure_lit()))
        return rc;
    CU(c, cudaEventRecord(x.ev_fork, x.st));
    int used = 0;
    cudaEvent_t e0 = profile ? prof_begin(c, x.st) : nullptr;
    for (int k = 0; k < kSwClasses; ++k) {
        if (!need[k])
            continue;
        cudaStream_t s = x.aux[used % kAux];
        CU(c, cudaStreamWaitEvent(s, x.ev_fork, 0));
        PairList pl{(const int32_t *)x.queue.p, 0, (const int64_t *)x.seg.p + 2 * k,
                    (int *)x.counters.p + kCounterStride * k};
        if (k != 4) {
            const int grid = c->sm_count * sw_blocks_per_sm(cls_band[k], var_of(cls_band[k]));
            CU(c, launch_sw(cls_band[k], var_of(cls_band[k]), qv, rv, p, cfg->band_width, d_bands,
                            pl, d_out, nullptr, 0, grid, s));
        } else {
            CU(c, launch_sw(0, 0, qv, rv, p, cfg->band_width, d_bands, pl, d_out,
                            (int64_t *)x.scratch64.p, lit_stride, lit_grid, s));
        }
        CU(c, cudaEventRecord(x.ev_join[used % kAux], s));
        ++used;
        c->launches += 1;
    }
    for (int i = 0; i < std::min(used, kAux); ++i)
        CU(c, cudaStreamWaitEvent(x.st, x.ev_join[i], 0));
    prof_end(c, e0, x.st);
    return GB2_OK;
}

int sw_validate(gb2_ctx *c, const gb2_sw_cfg *cfg, const int32_t *bands, int64_t n, int64_t qmax,
                int64_t rmax, SwPlanInfo &pi)
{
    if (!cfg)
        return set_err(c, GB2_EINVAL, "cfg is NULL");
    if (n < 0)
        return set_err(c, GB2_EINVAL, "n_pairs < 0");
    int32_t maxb = cfg->band_width;
    if (bands) {
        // one branch-free pass (it vectorises); the offending pair only on error
        int32_t lo = 0, hi = 0;
        for (int64_t i = 0; i < n; ++i) {
            lo = std::min(lo, bands[i]);
            hi = std::max(hi, bands[i]);
        }
        if (lo < 0) {
            int64_t i = 0;
            while (bands[i] >= 0)
                ++i;
            return set_err(c, GB2_EINVAL, "band of pair %lld is negative", (long long)i);
        }
        maxb = hi;
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
    const int32_t goe = cfg->gap_open + cfg->gap_extend;
    pi.pack_ok = pi.fast_ok && cfg->mismatch >= goe && cfg->match_score >= cfg->mismatch &&
                 cfg->match_score <= 255 && -goe <= 255 && -cfg->gap_extend <= 255 &&
                 cfg->match_score - cfg->mismatch <= 255;
    pi.wide_ok = pi.pack_ok && cfg->match_score <= 127;
    pi.max_band = maxb;
    pi.uniform_band = bands == nullptr;
    return GB2_OK;
}

// ---------------------------------------------------------------------------
// WFA core
// ---------------------------------------------------------------------------
static int gcd_h(int a, int b)
{
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

int wfa_validate(gb2_ctx *c, const gb2_wfa_cfg *cfg, int64_t n)
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

int wfa_begin(gb2_ctx *c, Exec &x)
{
    int rc;
    if ((rc = ensure(c, x.errflag, 64, x.st)) || (rc = ensure(c, x.work, 64, x.st)))
        return rc;
    CU(c, cudaMemsetAsync(x.errflag.p, 0, 64, x.st));
    CU(c, cudaMemsetAsync(x.work.p, 0, 64, x.st));
    return GB2_OK;
}

// Warps per block of the WFA kernel.  A batch of at most kWfaWideMaxPairs pairs (a
// request group of the server, a small call) that holds pairs of at least
// kWfaWideTeamLen bases runs the wide kernel: one 16-warp block per SM, each
// of those pairs aligned by a whole block, the rest one per warp.  A long
// pair's score steps are its critical path, so four times the threads per
// step cut a small batch's latency; large batches keep the 4-warp blocks,
// whose throughput is higher.
constexpr int64_t kWfaWideMaxPairs = 2048;
constexpr int64_t kWfaWideTeamLen = 8192;
static int wfa_block_warps(int64_t qmax, int64_t rmax, int64_t n, int variant)
{
    if (variant & 0xff)
        return 4;  // the tuning variants are 4-warp kernels
    return n <= kWfaWideMaxPairs && std::max(qmax, rmax) >= kWfaWideTeamLen ? kWfaWideWarps : 4;
}

// Tiered WFA (wfa_tiers.cu): every pair starts on the smallest team whose
// launch still fills the GPU -- one warp for large batches, four warps for up
// to 16 pairs per SM, eight for up to two per SM, sixteen for one, so a single
// long pair (the per-call drop-in) gets a whole SM -- and moves up a tier
// (1, 2, 4, 8, 16 warps) when its wavefront outgrows the window; pairs that
// outgrow the last or need int32 rows
// finish in G.  One launch per tier from the first, in order on x.st; the
// launches after the first take their pair count from the device.  With
// GB2_FLAG_BATCHED the first tier's queue is ordered longest first.
static int wfa_tiers(gb2_ctx *c, Exec &x, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
                     const WfaParams &p, int64_t n, int32_t *d_out, int flags, int32_t *d_ub)
{
    WfaTierPlan pl = wfa_tier_plan(p, qmax, rmax);
    const int64_t sms = c->sm_count;
    // The two-warp tier pays off when the batch leaves it enough pairs: on the
    // long-pair workload it saved 5 ms at 100,000 pairs and 1.4 ms at 40,000, and
    // cost 0.5 ms at 20,000 and 1.3 ms at 10,000 (one more launch in the chain).
    if (n < kWfaTwoWarpMinPairsPerSm * sms)
        pl.usable[1] = false;
    constexpr int G = kWfaShared;  // the global-memory tier
    int first = n <= sms ? 4 : (n <= 2 * sms ? 3 : (n <= 16 * sms ? 2 : 0));
    while (first < G && !pl.usable[first])
        ++first;
    auto next_of = [&](int t) {
        for (int u = t + 1; u < G; ++u)
            if (pl.usable[u])
                return u;
        return -1;
    };
    // dump records of the transitions out of the first two tiers
    int64_t dcap[G] = {}, doff[G] = {}, dbytes = 0;
    for (int t = first; t < G; ++t) {
        if (!pl.usable[t] || next_of(t) < 0)
            continue;
        dcap[t] = std::min<int64_t>(n, kTierDumpCap / pl.dump_stride[t]);
        doff[t] = dbytes;
        dbytes += dcap[t] * pl.dump_stride[t];
    }
    int rc;
    if ((rc = ensure(c, x.tierq, (size_t)n * 8 * G, x.st)) ||
        (rc = ensure(c, x.dumps, (size_t)std::max<int64_t>(dbytes, 256), x.st)) ||
        (rc = ensure(c, x.scratch32, (size_t)(sms * pl.gring_block_bytes), x.st)) ||
        (rc = ensure(c, x.counters, kCounterBytes, x.st)))
        return rc;
    CU(c, cudaMemsetAsync(x.counters.p, 0, kCounterBytes, x.st));
    int *const ctr = (int *)x.counters.p;
    int *const in_ctr = ctr;                             // + 32 * tier
    int *const q_n = ctr + (G + 1) * kCounterStride;     // + 32 * (tier - 1): pairs queued for tiers 1..G
    int *const d_ctr = ctr + (2 * G + 1) * kCounterStride;  // + 32 * tier: records claimed
    int *const b_ctr = ctr + (3 * G + 1) * kCounterStride;  // the bound pass
    static_assert((3 * G + 2) * kCounterStride * 4 <= (int)kCounterBytes, "counter space");
    int2 *const tq = (int2 *)x.tierq.p;              // + n * (tier - 1)
    uint8_t *const dumps = (uint8_t *)x.dumps.p;
    const int32_t *list = nullptr;
    const int64_t *seg = nullptr;
    if (flags & GB2_FLAG_BATCHED) {
        const int nb = kLenBuckets;
        if ((rc = ensure(c, x.keys, (size_t)n * 4, x.st)) ||
            (rc = ensure(c, x.queue, (size_t)n * 4, x.st)) ||
            (rc = ensure(c, x.counts, (size_t)nb * 4, x.st)) ||
            (rc = ensure(c, x.seg, 64, x.st)))
            return rc;
        CU(c, cudaMemsetAsync(x.counts.p, 0, (size_t)nb * 4, x.st));
        const int blocks = (int)((n + 255) / 256);
        k_classify_wfa<<<blocks, 256, 0, x.st>>>(n, qv, rv, (int32_t *)x.keys.p,
                                                  (int *)x.counts.p);
        k_scan<<<1, 1024, 0, x.st>>>((int *)x.counts.p, nb, nb, (int64_t *)x.seg.p);
        k_scatter<<<blocks, 256, 0, x.st>>>(n, (const int32_t *)x.keys.p, (int *)x.counts.p,
                                             (int32_t *)x.queue.p);
        CU(c, cudaGetLastError());
        c->launches += 3;
        list = (const int32_t *)x.queue.p;
        seg = (const int64_t *)x.seg.p;
    }
    static const int teams_per_block[G + 1] = {16, 8, 4, 2, 1, 1};
    int prev = -1;  // the tier launched before t: its suspended pairs are t's entries
    for (int t = first; t <= G; ++t) {
        if (t < G && !pl.usable[t])
            continue;
        WfaTierIo io{};
        io.ctr = in_ctr + kCounterStride * t;
        if (t == first) {
            io.list = list;
            io.seg = seg;
            io.n = n;
        } else {
            io.ents = tq + n * (t - 1);
            io.n_dev = q_n + kCounterStride * (t - 1);
            if (t < G && prev >= 0 && dcap[prev] > 0) {  // G entries always start over
                io.dumps_in = dumps + doff[prev];
                io.dump_in_stride = pl.dump_stride[prev];
            }
        }
        const int nt = t < G ? next_of(t) : -1;
        if (nt >= 0) {
            io.next = tq + n * (nt - 1);
            io.next_n = q_n + kCounterStride * (nt - 1);
            io.dumps_out = dumps + doff[t];
            io.dump_out_stride = pl.dump_stride[t];
            io.dump_out_cap = dcap[t];
            io.dump_out_ctr = d_ctr + kCounterStride * t;
        }
        if (t < G) {
            io.restart = tq + n * (G - 1);
            io.restart_n = q_n + kCounterStride * (G - 1);
        }
        io.gring = (int32_t *)x.scratch32.p;
        // the tiers after the first prune by the bound pass's costs
        io.ubound = (d_ub && t > 0) ? d_ub : nullptr;
        const int64_t per = teams_per_block[t];
        const int grid = (int)(t == first ? std::min<int64_t>(sms, (n + per - 1) / per) : sms);
        cudaEvent_t e0 = prof_begin(c, x.st);
        CU(c, launch_wfa_tier(pl, t, grid, qv, rv, p, io, d_out, (int64_t *)x.work.p,
                              (int *)x.errflag.p, x.st));
        prof_end(c, e0, x.st);
        c->launches += 1;
        if (t == 0 && d_ub && nt >= 0) {
            // The bound pass: the pairs the one-warp tier suspended continue from
            // their records (read, not consumed) on the one-warp kernel inside a band of
            // +-kWfaBoundBand diagonals around the line from diagonal 0 to the
            // target.  A hit there is a real alignment, so its cost bounds the
            // optimum from above; a pair the band cannot finish gets -1 (the
            // bound is then max_error).
            WfaTierIo bp{};
            bp.ctr = b_ctr;
            bp.ents = io.next;
            bp.n_dev = io.next_n;
            bp.dumps_in = io.dumps_out;
            bp.dump_in_stride = io.dump_out_stride;
            bp.band_w = kWfaBoundBand;
            bp.gring = io.gring;
            cudaEvent_t e1 = prof_begin(c, x.st);
            CU(c, launch_wfa_tier(pl, 0, (int)sms, qv, rv, p, bp, d_ub, (int64_t *)x.work.p,
                                  (int *)x.errflag.p, x.st));
            prof_end(c, e1, x.st);
            c->launches += 1;
        }
        prev = t;
    }
    return GB2_OK;
}

int wfa_core(gb2_ctx *c, Exec &x, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
             const gb2_wfa_cfg *cfg, int64_t n, int32_t *d_out, int flags, int64_t *d_hist)
{
    if (n <= 0)
        return GB2_OK;
    if (qmax >= (1ll << 30) || rmax >= (1ll << 30))
        return set_err(c, GB2_ERANGE, "sequence longer than 2^30");
    const WfaParams p{cfg->x, cfg->o, cfg->e, cfg->max_error};
    // the tiered kernels, unless the call asks for the naive baseline, a tuning
    // variant of the single-kernel design below, or the CIGAR pass's history sizes
    if (!(flags & GB2_FLAG_NAIVE) && ((flags >> 8) & 0xff) == 0 && !d_hist) {
        // Batches with long pairs: for every pair the one-warp tier suspends (the
        // expensive ones), a bound pass finds the cost of its best alignment
        // inside a band of +-kWfaBoundBand diagonals around the line from
        // diagonal 0 to the target -- the cost of a real alignment, so no lower
        // than the optimum -- and the later tiers skip every diagonal that cannot
        // finish within it (s + e*|k - target| > bound): the same costs, far
        // fewer cells where the wavefronts are widest.
        if ((flags & GB2_FLAG_NO_PRUNE) || std::max(qmax, rmax) < kWfaBoundMinLen)
            return wfa_tiers(c, x, qv, rv, qmax, rmax, p, n, d_out, flags, nullptr);
        int rc;
        if ((rc = ensure(c, x.ubound, (size_t)n * 4, x.st)))
            return rc;
        CU(c, cudaMemsetAsync(x.ubound.p, 0xff, (size_t)n * 4, x.st));  // -1: no bound yet
        return wfa_tiers(c, x, qv, rv, qmax, rmax, p, n, d_out, flags, (int32_t *)x.ubound.p);
    }
    const int g = gcd_h(cfg->x, gcd_h(cfg->o, cfg->e));
    const int hm = std::max(cfg->x / g, (cfg->o + cfg->e) / g) + 1, hie = cfg->e / g + 1;
    const int nslot = hm + 2 * hie;
    const int64_t slot_width = ((qmax + rmax + 5) + 31) & ~int64_t(31);
    // blocks of 4 warps, as many per SM as stay resident, fewer when the rings
    // of that many warps would pass kWfaScratchCap bytes.  Tuning knob in
    // flags bits 8-15: low 4 bits = blocks per SM, bits 4-5 = kernel unroll
    // choice, bit 6 = no pair aligned by a whole block, bit 7 = every pair of
    // at least kWfaTeamMinLen bases aligned by a whole block.
    const int fvar = (flags >> 8) & 0xff;
    const int bw = wfa_block_warps(qmax, rmax, n, fvar);
    // the caller's variant, else (4-warp kernel) the one installed by the tuner
    const int variant = fvar ? fvar : (bw == 4 ? c->tune_wfa : 0);
    const int64_t warp_bytes = (int64_t)nslot * slot_width * 4;
    int64_t grid = (int64_t)c->sm_count *
                   ((variant & 15) ? (variant & 15) : wfa_blocks_per_sm(variant, bw));
    grid = std::min(grid, std::max<int64_t>(c->sm_count, kWfaScratchCap / (bw * warp_bytes)));
    // a plain batch of at most one wave of blocks (a per-call drop-in) runs one
    // block per pair (below); otherwise no more blocks than the warps need
    const bool plain_blocks = !(flags & GB2_FLAG_BATCHED) && n <= grid;
    // the naive baseline: every pair, in input order, by a whole block (blocks
    // take the next pair when done, so the rings stay one region per block)
    const bool naive = (flags & GB2_FLAG_NAIVE) != 0;
    grid = plain_blocks ? n
                        : std::min(grid, std::max<int64_t>(1, (bw == 4 && !naive) ? (n + 3) / 4 : n));
    int rc;
    if ((rc = ensure(c, x.scratch32, (size_t)(grid * bw * warp_bytes), x.st)) ||
        (rc = ensure(c, x.counters, kCounterBytes, x.st)))
        return rc;
    CU(c, cudaMemsetAsync(x.counters.p, 0, kCounterBytes, x.st));
    int *const ctr = (int *)x.counters.p;
    PairList longs{nullptr, 0, nullptr, ctr + kCounterStride};
    PairList shorts{nullptr, n, nullptr, ctr};
    if (plain_blocks || naive) {
        // every pair, in input order, is aligned by a whole block, so a long pair's
        // score steps are shared by the block's warps instead of running on one warp
        longs = PairList{nullptr, n, nullptr, ctr + kCounterStride};
        shorts = PairList{nullptr, 0, nullptr, ctr};
    }
    if ((flags & GB2_FLAG_BATCHED) && !naive) {
        const int nb = kLenBuckets;
        // one pair per block for the longest pairs: one wave of blocks of them, or
        // with the wide kernel every pair of at least kWfaWideTeamLen bases
        const int64_t team_pairs =
            (variant & 0x40) ? 0 : ((variant & 0x80) || bw != 4) ? n : grid;
        const int64_t team_len = bw != 4 ? kWfaWideTeamLen : kWfaTeamMinLen;
        if ((rc = ensure(c, x.keys, (size_t)n * 4, x.st)) ||
            (rc = ensure(c, x.queue, (size_t)n * 4, x.st)) ||
            (rc = ensure(c, x.counts, (size_t)nb * 4, x.st)) ||
            (rc = ensure(c, x.seg, 64, x.st)))
            return rc;
        CU(c, cudaMemsetAsync(x.counts.p, 0, (size_t)nb * 4, x.st));
        const int blocks = (int)((n + 255) / 256);
        int64_t *seg = (int64_t *)x.seg.p;
        k_classify_wfa<<<blocks, 256, 0, x.st>>>(n, qv, rv, (int32_t *)x.keys.p,
                                                  (int *)x.counts.p);
        k_scan<<<1, 1024, 0, x.st>>>((int *)x.counts.p, nb, nb, seg);
        k_split_wfa<<<1, 1, 0, x.st>>>((const int *)x.counts.p, n, team_len, team_pairs, seg);
        k_scatter<<<blocks, 256, 0, x.st>>>(n, (const int32_t *)x.keys.p, (int *)x.counts.p,
                                             (int32_t *)x.queue.p);
        CU(c, cudaGetLastError());
        c->launches += 4;
        const int32_t *qd = (const int32_t *)x.queue.p;
        longs = PairList{qd, 0, seg, ctr + kCounterStride};
        shorts = PairList{qd, 0, seg + 2, ctr};
    }
    cudaEvent_t e0 = prof_begin(c, x.st);
    CU(c, launch_wfa(variant, bw, qv, rv, p, longs, shorts, d_out, (int32_t *)x.scratch32.p,
                     slot_width, (int)grid, (int *)x.errflag.p, (int64_t *)x.work.p, d_hist,
                     x.st));
    prof_end(c, e0, x.st);
    c->launches += 1;
    return GB2_OK;
}

int wfa_end(gb2_ctx *c, Exec &x)
{
    int flag = 0;
    int64_t work = 0;
    CU(c, cudaMemcpyAsync(&flag, x.errflag.p, 4, cudaMemcpyDeviceToHost, x.st));
    CU(c, cudaMemcpyAsync(&work, x.work.p, 8, cudaMemcpyDeviceToHost, x.st));
    CU(c, cudaStreamSynchronize(x.st));
    c->work_units += work;
    if (flag)
        return set_err(c, GB2_EKERNEL, "WFA kernel reported a pair longer than its scratch");
    return GB2_OK;
}

}  // namespace gb2

// ---------------------------------------------------------------------------
// blocking helpers of the context's own executor
// ---------------------------------------------------------------------------
static SeqView view_of(const gb2_batch *b)
{
    return SeqView{b->d_packed, b->d_offsets, b->d_lengths, 0, std::max<int64_t>(b->n_words, 1)};
}

static int sync_and_check(gb2_ctx *c)
{
    CU(c, cudaStreamSynchronize(c->x.st));
    harvest_profile(c);
    return GB2_OK;
}

// Runs a resident call's device work on c->x.st, eagerly or, with
// GB2_FLAG_GRAPH, through the context's replay cache g (GraphCache): the
// first call with a key runs eagerly, the second is captured into a CUDA
// graph, later ones launch it.  Eager is the default: each call here is one
// to five persistent launches, and replaying them from a graph measured 6-10%
// slower per call than launching them (2,000 mixed-band pairs: 3.04 vs
// 2.75 ms; 5,000 reads: 164 vs 155 us).
// issue(capturing) enqueues the work, joins every other stream it forks back
// into c->x.st, and writes to the host only by cudaMemcpyAsync into the
// pinned array at `host` (nullptr: no host copies in the work).  While
// profiling is on, calls run eagerly: the kernel spans need events between
// the launches, which a graph does not hold.  A capture that fails (an
// unexpected reallocation, an unsupported call) leaves the key eager.
template <typename Issue>
static int run_graphed(gb2_ctx *c, GraphCache &g, const std::vector<int64_t> &key, int flags,
                       char *host, Issue issue)
{
    if (!(flags & GB2_FLAG_GRAPH) || c->profiling.load())
        return issue(false);
    if (g.key != key || g.gen != c->buf_gen) {  // first call with this shape
        g.reset();
        g.key = key;
        const int rc = issue(false);
        g.gen = c->buf_gen;  // the call's own allocations belong to the shape
        return rc;
    }
    if (g.failed)
        return issue(false);
    if (!g.exec) {
        const int64_t l0 = c->launches.load();
        cudaGraph_t graph = nullptr;
        int rc = GB2_ECUDA;
        if (cudaStreamBeginCapture(c->x.st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            rc = issue(true);
            if (cudaStreamEndCapture(c->x.st, &graph) != cudaSuccess && rc == GB2_OK)
                rc = GB2_ECUDA;
        }
        c->launches = l0;
        bool ok = rc == GB2_OK && graph && c->buf_gen == g.gen &&
                  cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess;
        if (ok) {
            size_t nn = 0;
            ok = cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess;
            std::vector<cudaGraphNode_t> nodes(nn);
            ok = ok && cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess;
            for (size_t i = 0; ok && i < nn; ++i) {
                cudaGraphNodeType t;
                ok = cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess;
                if (ok && t == cudaGraphNodeTypeKernel) {
                    ++g.kernels;
                } else if (ok && t == cudaGraphNodeTypeMemcpy) {
                    cudaMemcpy3DParms mp{};
                    ok = cudaGraphMemcpyNodeGetParams(nodes[i], &mp) == cudaSuccess;
                    const char *dst = (const char *)mp.dstPtr.ptr;
                    ok = ok && host && mp.kind == cudaMemcpyDeviceToHost && dst >= host &&
                         mp.extent.height <= 1 && mp.extent.depth <= 1;
                    if (ok)
                        g.copies.push_back(GraphCache::Copy{nodes[i], (size_t)(dst - host),
                                                            mp.extent.width, mp.srcPtr.ptr});
                }
            }
        }
        if (!ok) {
            if (g.exec)
                cudaGraphExecDestroy(g.exec);
            if (graph)
                cudaGraphDestroy(graph);
            g.exec = nullptr;
            g.copies.clear();
            g.kernels = 0;
            g.failed = true;
            cudaGetLastError();
            return issue(false);
        }
        g.graph = graph;
        g.host = host;
    }
    if (host != g.host) {  // the caller's result array moved: retarget the copies
        for (const GraphCache::Copy &cp : g.copies)
            if (cudaGraphExecMemcpyNodeSetParams1D(g.exec, cp.node, host + cp.dst_off, cp.src,
                                                    cp.bytes, cudaMemcpyDeviceToHost) !=
                cudaSuccess) {
                g.reset();
                cudaGetLastError();
                return issue(false);
            }
        g.host = host;
    }
    CU(c, cudaGraphLaunch(g.exec, c->x.st));
    c->launches += g.kernels;
    return GB2_OK;
}

// The shape of a resident call over batches q and r, for GraphCache keys.
static void key_batches(std::vector<int64_t> &k, const gb2_batch *q, const gb2_batch *r)
{
    for (const gb2_batch *b : {q, r}) {
        k.push_back((int64_t)(uintptr_t)b->d_packed);
        k.push_back((int64_t)(uintptr_t)b->d_offsets);
        k.push_back((int64_t)(uintptr_t)b->d_lengths);
        k.push_back(b->count);
        k.push_back(b->n_words);
        k.push_back(b->max_len);
        k.push_back(b->min_len);
    }
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
    CU(c, pinned_alloc(&c->pin_out, bytes));
    c->pin_out_cap = bytes;
    return GB2_OK;
}

static int d2h_results(gb2_ctx *c, void *host, const void *dev, size_t bytes)
{
    if (bytes == 0)
        return GB2_OK;
    if (is_pinned(host)) {
        CU(c, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->x.st));
        return sync_and_check(c);
    }
    int rc = pin_out(c, bytes);
    if (rc)
        return rc;
    CU(c, cudaMemcpyAsync(c->pin_out, dev, bytes, cudaMemcpyDeviceToHost, c->x.st));
    if ((rc = sync_and_check(c)))
        return rc;
    memcpy(host, c->pin_out, bytes);
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

// One host pass over a chunk's pairs, per side: the word range the chunk's
// sequences occupy ([smallest offset, largest end), so any layout works --
// add_sequence's append layout (genomics/core/sequence.mojo:44-66) makes it
// the chunk's own contiguous run of words), the longest and shortest
// sequence, whether any offset or length is negative, and whether every
// sequence starts at the word where the previous one ends (then the offsets
// follow from the lengths and are not copied: the lengths are written here
// as int32 into pinned staging, and the device rebuilds both int64 arrays).
// Large chunks are split over two threads.
struct ChunkScan {
    int64_t qw0, qw1, rw0, rw1, qmaxlen, rmaxlen;
    bool negative, narrow;  // narrow: every length within narrow_range
    bool dense;             // both sides contiguous, lengths staged as int32
};

static void scan_side(const HostSide &h, int64_t i0, int64_t i1, int64_t &w0, int64_t &w1,
                      int64_t &minlen, int64_t &maxlen, int64_t &bits, bool &contig,
                      int32_t *len32)
{
    int64_t lo = INT64_MAX, hi = 0, mn = INT64_MAX, mx = 0, b = 0;
    int64_t expect = i1 > i0 ? h.offsets[i0] : 0;
    bool ct = true;
    for (int64_t i = i0; i < i1; ++i) {
        const int64_t o = h.offsets[i], l = h.lengths[i];
        b |= o | l;
        mx = l > mx ? l : mx;
        mn = l < mn ? l : mn;
        lo = o < lo ? o : lo;
        const int64_t e = o + ((l + 31) >> 5);
        hi = e > hi ? e : hi;
        ct &= o == expect;
        expect = e;
        len32[i - i0] = (int32_t)l;
    }
    w0 = lo;
    w1 = hi;
    minlen = mn;
    maxlen = mx;
    bits = b;
    contig = ct;
}

// One side's part of a chunk scan.
struct SideScan {
    int64_t w0 = 0, w1 = 0, minlen = 0, maxlen = 0, bits = 0;
    bool contig = true;
};

static ChunkScan combine(const SideScan &q, const SideScan &r)
{
    ChunkScan o;
    o.negative = (q.bits | r.bits) < 0;
    o.qw0 = q.w0;
    o.qw1 = std::max(q.w1, q.w0);
    o.rw0 = r.w0;
    o.rw1 = std::max(r.w1, r.w0);
    o.qmaxlen = q.maxlen;
    o.rmaxlen = r.maxlen;
    o.narrow = narrow_range(q.minlen, q.maxlen) && narrow_range(r.minlen, r.maxlen);
    o.dense = q.contig && r.contig && q.maxlen < (1ll << 31) && r.maxlen < (1ll << 31);
    return o;
}

// Rebuilds a contiguous chunk's int64 offsets and lengths from its int32
// lengths: offsets[i] = base + sum of words(lengths[j]) over j < i.  Two
// launches over tiles of kExpandTile pairs (256 threads x 8 consecutive pairs,
// coalesced): k_expand_sums writes each tile's word totals, k_expand_write
// adds the totals of the tiles before its own to a block-wide scan and writes
// both arrays.
constexpr int kExpandTile = 2048;

__device__ __forceinline__ int64_t block_sum_256(int64_t v, int64_t *sh)
{
    for (int o = 16; o; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = v;
    __syncthreads();
    int64_t t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < 8 ? sh[threadIdx.x] : 0;
        for (int o = 4; o; o >>= 1)
            t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

__global__ void __launch_bounds__(256)
k_expand_sums(int64_t m, const int32_t *__restrict__ q32, const int32_t *__restrict__ r32,
              int64_t *__restrict__ sums)
{
    __shared__ int64_t sh[8];
    const int64_t i0 = (int64_t)blockIdx.x * kExpandTile + threadIdx.x * 8;
    int64_t aq = 0, ar = 0;
    for (int k = 0; k < 8; ++k) {
        const int64_t i = i0 + k;
        if (i < m) {
            aq += ((int64_t)q32[i] + 31) >> 5;
            ar += ((int64_t)r32[i] + 31) >> 5;
        }
    }
    const int64_t tq = block_sum_256(aq, sh);
    const int64_t tr = block_sum_256(ar, sh);
    if (threadIdx.x == 0) {
        sums[2 * blockIdx.x] = tq;
        sums[2 * blockIdx.x + 1] = tr;
    }
}

__global__ void __launch_bounds__(256)
k_expand_write(int64_t m, const int32_t *__restrict__ q32, const int32_t *__restrict__ r32,
               const int64_t *__restrict__ sums, int64_t qbase, int64_t rbase,
               int64_t *__restrict__ qo, int64_t *__restrict__ ql, int64_t *__restrict__ ro,
               int64_t *__restrict__ rl)
{
    __shared__ int64_t sh[8];
    __shared__ int64_t wq[8], wr[8];
    // totals of the tiles before this one
    int64_t pq = 0, pr = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) {
        pq += sums[2 * b];
        pr += sums[2 * b + 1];
    }
    pq = block_sum_256(pq, sh);
    pr = block_sum_256(pr, sh);
    __shared__ int64_t base_q, base_r;
    if (threadIdx.x == 0) {
        base_q = qbase + pq;
        base_r = rbase + pr;
    }
    // this thread's 8 pairs, then an exclusive scan over the block
    const int64_t i0 = (int64_t)blockIdx.x * kExpandTile + threadIdx.x * 8;
    int32_t lq[8], lr[8];
    int64_t aq = 0, ar = 0;
    for (int k = 0; k < 8; ++k) {
        const int64_t i = i0 + k;
        lq[k] = i < m ? q32[i] : 0;
        lr[k] = i < m ? r32[i] : 0;
        aq += ((int64_t)lq[k] + 31) >> 5;
        ar += ((int64_t)lr[k] + 31) >> 5;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t xq = aq, xr = ar;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t vq = __shfl_up_sync(0xffffffffu, xq, o);
        const int64_t vr = __shfl_up_sync(0xffffffffu, xr, o);
        if (lane >= o) {
            xq += vq;
            xr += vr;
        }
    }
    if (lane == 31) {
        wq[warp] = xq;
        wr[warp] = xr;
    }
    __syncthreads();
    int64_t oq = base_q + xq - aq, orr = base_r + xr - ar;
    for (int w = 0; w < warp; ++w) {
        oq += wq[w];
        orr += wr[w];
    }
    for (int k = 0; k < 8; ++k) {
        const int64_t i = i0 + k;
        if (i < m) {
            qo[i] = oq;
            ql[i] = lq[k];
            ro[i] = orr;
            rl[i] = lr[k];
        }
        oq += ((int64_t)lq[k] + 31) >> 5;
        orr += ((int64_t)lr[k] + 31) >> 5;
    }
}

// Grows the context's pinned int32 length staging of the host pipeline.
static int ensure_len32(gb2_ctx *c, size_t bytes)
{
    if (bytes <= c->pin_len32_cap)
        return GB2_OK;
    if (c->pin_len32)
        cudaFreeHost(c->pin_len32);
    c->pin_len32 = nullptr;
    c->pin_len32_cap = 0;
    const size_t cap = std::max<size_t>(bytes + bytes / 4, 1 << 16);
    CU(c, pinned_alloc(&c->pin_len32, cap));
    c->pin_len32_cap = cap;
    return GB2_OK;
}

// Chunked host-to-device pipeline.  For each chunk the host scans the
// chunk's offsets and lengths (while the GPU copies and aligns earlier
// chunks), copies the word range the chunk touches plus its lengths (int32,
// offsets rebuilt on the device by two small kernels on a stream of their
// own, when the chunk is contiguous; else int64 offsets and lengths) and
// bands on the copy stream, and runs the chunk on one of the context's two
// executors (alternating, so one chunk's kernels can fill the GPU while the
// previous chunk's last blocks drain); results come back on a separate
// stream, so an executor's stream holds nothing but alignment kernels.
// kPipeSets chunks are in flight: the copies of a chunk wait on the device for
// the chunk that last used its buffers.  On any error every stream is drained before returning, so no copy
// touches the caller's memory after the call.
template <typename RunChunk>
static int pipeline(gb2_ctx *c, const HostSide &hq, const HostSide &hr, const int32_t *bands,
                    int64_t n, size_t out_elem, void *out_host, int64_t chunk_pairs,
                    RunChunk run_chunk)
{
    std::vector<int64_t> bounds{0};
    while (bounds.back() < n)
        bounds.push_back(std::min(n, bounds.back() + chunk_pairs));
    const int64_t nchunks = (int64_t)bounds.size() - 1;
    int rc = GB2_OK;
    const bool out_pinned = is_pinned(out_host);
    if (!out_pinned && (rc = pin_out(c, (size_t)n * out_elem)))
        return rc;
    // Two scanner threads (one per side) run through all chunks ahead of the
    // issuing thread, writing each chunk's int32 lengths into pinned staging
    // (chunk [p0, p1): q at 2*p0, r right after) and publishing the chunk's
    // scan; the issuing thread waits only for chunks not scanned yet.  The
    // staging is the context's and is free: the previous call's copies ended
    // before it returned.
    if ((rc = ensure_len32(c, (size_t)n * 8)))
        return rc;
    int32_t *const stage = (int32_t *)c->pin_len32;
    std::vector<SideScan> sq((size_t)nchunks), sr((size_t)nchunks);
    std::atomic<int64_t> q_done{0}, r_done{0};
    auto scanner = [&](const HostSide &h, std::vector<SideScan> *out, std::atomic<int64_t> *done,
                       int side) {
        for (int64_t ci = 0; ci < nchunks; ++ci) {
            const int64_t p0 = bounds[(size_t)ci], p1 = bounds[(size_t)ci + 1];
            SideScan &sc = (*out)[(size_t)ci];
            scan_side(h, p0, p1, sc.w0, sc.w1, sc.minlen, sc.maxlen, sc.bits, sc.contig,
                      stage + 2 * p0 + (side ? p1 - p0 : 0));
            done->store(ci + 1, std::memory_order_release);
        }
    };
    // a small batch (a per-call drop-in among them) is scanned on this thread:
    // starting two threads would cost more than the scan
    const bool inline_scan = n <= kInlineScanPairs;
    std::thread tq, tr;
    if (inline_scan) {
        scanner(hq, &sq, &q_done, 0);
        scanner(hr, &sr, &r_done, 1);
    } else {
        tq = std::thread(scanner, std::cref(hq), &sq, &q_done, 0);
        tr = std::thread(scanner, std::cref(hr), &sr, &r_done, 1);
    }
    struct Joiner {
        std::thread &a, &b;
        ~Joiner()
        {
            if (a.joinable())
                a.join();
            if (b.joinable())
                b.join();
        }
    } joiner{tq, tr};
    auto issue = [&](int64_t ci) -> int {
        PipeSet &ps = c->pipe[ci % kPipeSets];
        Exec &x = (ci & 1) ? c->x2 : c->x;
        const int64_t p0 = bounds[(size_t)ci], p1 = bounds[(size_t)ci + 1];
        const int64_t m = p1 - p0;
        int r;
        while (q_done.load(std::memory_order_acquire) <= ci ||
               r_done.load(std::memory_order_acquire) <= ci)
            std::this_thread::yield();
        int32_t *q32 = stage + 2 * p0;
        const ChunkScan cs = combine(sq[(size_t)ci], sr[(size_t)ci]);
        if (cs.negative)
            return set_err(c, GB2_EINVAL, "negative offset or length among pairs %lld-%lld",
                           (long long)p0, (long long)(p1 - 1));
        const int64_t qn = std::max<int64_t>(cs.qw1 - cs.qw0, 1);
        const int64_t rn = std::max<int64_t>(cs.rw1 - cs.rw0, 1);
        const bool grow = ps.qw.cap < (size_t)qn * 8 || ps.rw.cap < (size_t)rn * 8 ||
                          ps.qo.cap < (size_t)m * 8 || ps.out.cap < (size_t)m * out_elem ||
                          ps.len32.cap < (size_t)m * 8 + 16 * (m / kExpandTile + 1) ||
                          (bands && ps.bands.cap < (size_t)m * 4);
        if (grow)  // reallocating: the set's previous chunk must be completely done
            CU(c, cudaEventSynchronize(ps.done));
        if ((r = ensure(c, ps.qw, qn * 8, x.st)) || (r = ensure(c, ps.rw, rn * 8, x.st)) ||
            (r = ensure(c, ps.qo, m * 8, x.st)) || (r = ensure(c, ps.ql, m * 8, x.st)) ||
            (r = ensure(c, ps.ro, m * 8, x.st)) || (r = ensure(c, ps.rl, m * 8, x.st)) ||
            (r = ensure(c, ps.out, m * out_elem, x.st)) ||
            (r = ensure(c, ps.len32, m * 8 + 16 * (m / kExpandTile + 1), x.st)) ||
            (bands && (r = ensure(c, ps.bands, m * 4, x.st))))
            return r;
        // the device buffers of this set's previous chunk are free once it is done
        CU(c, cudaStreamWaitEvent(c->st_copy, ps.done, 0));
        if ((r = h2d(c, ps.qw.p, hq.packed + cs.qw0, (size_t)(cs.qw1 - cs.qw0) * 8, c->st_copy)) ||
            (r = h2d(c, ps.rw.p, hr.packed + cs.rw0, (size_t)(cs.rw1 - cs.rw0) * 8, c->st_copy)))
            return r;
        if (cs.dense) {
            CU(c, cudaMemcpyAsync(ps.len32.p, q32, (size_t)m * 8, cudaMemcpyHostToDevice,
                                  c->st_copy));
        } else if ((r = h2d(c, ps.qo.p, hq.offsets + p0, (size_t)m * 8, c->st_copy)) ||
                   (r = h2d(c, ps.ql.p, hq.lengths + p0, (size_t)m * 8, c->st_copy)) ||
                   (r = h2d(c, ps.ro.p, hr.offsets + p0, (size_t)m * 8, c->st_copy)) ||
                   (r = h2d(c, ps.rl.p, hr.lengths + p0, (size_t)m * 8, c->st_copy))) {
            return r;
        }
        if (bands && (r = h2d(c, ps.bands.p, bands + p0, (size_t)m * 4, c->st_copy)))
            return r;
        CU(c, cudaEventRecord(ps.copied, c->st_copy));
        if (cs.dense) {  // rebuild the offsets beside the executors, off the copy stream
            CU(c, cudaStreamWaitEvent(c->st_prep, ps.copied, 0));
            const int32_t *d32 = (const int32_t *)ps.len32.p;
            int64_t *sums = (int64_t *)((char *)ps.len32.p + (size_t)m * 8);
            const int tiles = (int)((m + kExpandTile - 1) / kExpandTile);
            k_expand_sums<<<tiles, 256, 0, c->st_prep>>>(m, d32, d32 + m, sums);
            k_expand_write<<<tiles, 256, 0, c->st_prep>>>(m, d32, d32 + m, sums, cs.qw0, cs.rw0,
                                                          (int64_t *)ps.qo.p, (int64_t *)ps.ql.p,
                                                          (int64_t *)ps.ro.p, (int64_t *)ps.rl.p);
            CU(c, cudaGetLastError());
            c->launches += 2;
            CU(c, cudaEventRecord(ps.ready, c->st_prep));
            CU(c, cudaStreamWaitEvent(x.st, ps.ready, 0));
        } else {
            CU(c, cudaStreamWaitEvent(x.st, ps.copied, 0));
        }
        const SeqView qv{(const uint64_t *)ps.qw.p, (const int64_t *)ps.qo.p,
                         (const int64_t *)ps.ql.p, cs.qw0, qn};
        const SeqView rv{(const uint64_t *)ps.rw.p, (const int64_t *)ps.ro.p,
                         (const int64_t *)ps.rl.p, cs.rw0, rn};
        if ((r = run_chunk(x, qv, rv, cs.qmaxlen, cs.rmaxlen, cs.narrow,
                           bands ? (const int32_t *)ps.bands.p : nullptr,
                           bands ? bands + p0 : nullptr, m, ps.out.p)))
            return r;
        void *dst = out_pinned ? (char *)out_host + p0 * out_elem
                               : (char *)c->pin_out + p0 * out_elem;
        // results return on their own stream, so the executor's next chunk does not
        // wait for this copy
        CU(c, cudaEventRecord(ps.kern, x.st));
        CU(c, cudaStreamWaitEvent(c->st_back, ps.kern, 0));
        CU(c, cudaMemcpyAsync(dst, ps.out.p, (size_t)m * out_elem, cudaMemcpyDeviceToHost,
                              c->st_back));
        CU(c, cudaEventRecord(ps.done, c->st_back));
        return GB2_OK;
    };
    for (int64_t ci = 0; ci < nchunks && !rc; ++ci)
        rc = issue(ci);
    if (rc) {
        for (cudaStream_t st : {c->st_copy, c->st_prep, c->x.st, c->x2.st, c->st_back})
            cudaStreamSynchronize(st);
        cudaGetLastError();
        return rc;
    }
    CU(c, cudaStreamSynchronize(c->x2.st));
    CU(c, cudaStreamSynchronize(c->st_back));
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

int gb2_debug_fail_alloc(int kind, int64_t nth)
{
    if (kind != GB2_ALLOC_DEVICE && kind != GB2_ALLOC_PINNED)
        return GB2_EINVAL;
    (kind == GB2_ALLOC_DEVICE ? g_fail_dev : g_fail_pin).store(nth < 0 ? -1 : nth);
    return GB2_OK;
}

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
    case GB2_ECANCELED: return "cancelled";
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
    bool ok = exec_init(c->x) == GB2_OK && exec_init(c->x2) == GB2_OK &&
              cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->st_prep, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->st_back, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&c->t0) == cudaSuccess && cudaEventCreate(&c->t1) == cudaSuccess;
    for (int i = 0; ok && i < 2; ++i) {
        ok = pinned_alloc(&c->pin[i], (size_t)kPinChunk) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->pin_ev[i], cudaEventDisableTiming) == cudaSuccess;
        if (ok)
            cudaEventRecord(c->pin_ev[i], c->x.st);
    }
    for (int i = 0; ok && i < kResidentParts; ++i)
        ok = cudaEventCreateWithFlags(&c->kdone[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->ev_join2, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < kPipeSets; ++i) {
        PipeSet &ps = c->pipe[i];
        for (cudaEvent_t *e : {&ps.copied, &ps.ready, &ps.kern, &ps.done}) {
            ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
            if (ok)
                cudaEventRecord(*e, c->x.st);
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
    for (cudaStream_t st : {c->st_copy, c->st_prep, c->st_back, c->x.st, c->x2.st})
        if (st)
            cudaStreamSynchronize(st);
    harvest_profile(c);
    c->g_sw.reset();
    c->g_wfa.reset();
    exec_free(c->x);
    exec_free(c->x2);
    CigarBufs &cb = c->cig;
    DevBuf *bufs[] = {&c->out_sw,     &c->out_wfa,  &c->bands,     &c->flush,
                      &cb.cost,       &cb.hist,     &cb.pairs,     &cb.arena_off,
                      &cb.arena,      &cb.runs,     &cb.run_off,   &cb.run_count,
                      &cb.out_off,    &cb.out};
    for (DevBuf *b : bufs)
        if (b->p)
            cudaFree(b->p);
    for (int i = 0; i < kPipeSets; ++i) {
        PipeSet &ps = c->pipe[i];
        DevBuf *pb[] = {&ps.qw, &ps.rw,    &ps.qo,  &ps.ql,   &ps.ro,
                        &ps.rl, &ps.bands, &ps.out, &ps.len32};
        for (DevBuf *b : pb)
            if (b->p)
                cudaFree(b->p);
        for (cudaEvent_t e : {ps.copied, ps.ready, ps.kern, ps.done})
            if (e)
                cudaEventDestroy(e);
    }
    for (int i = 0; i < kResidentParts; ++i)
        if (c->kdone[i])
            cudaEventDestroy(c->kdone[i]);
    if (c->ev_join2)
        cudaEventDestroy(c->ev_join2);
    for (int i = 0; i < 2; ++i) {
        if (c->pin[i])
            cudaFreeHost(c->pin[i]);
        if (c->pin_ev[i])
            cudaEventDestroy(c->pin_ev[i]);
    }
    if (c->pin_out)
        cudaFreeHost(c->pin_out);
    if (c->pin_len32)
        cudaFreeHost(c->pin_len32);
    if (c->t0)
        cudaEventDestroy(c->t0);
    if (c->t1)
        cudaEventDestroy(c->t1);
    for (cudaStream_t st : {c->st_copy, c->st_prep, c->st_back})
        if (st)
            cudaStreamDestroy(st);
    delete c;
    return GB2_OK;
}

int gb2_sync(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    for (cudaStream_t st : {c->st_copy, c->st_prep, c->st_back, c->x2.st})
        CU(c, cudaStreamSynchronize(st));
    return sync_and_check(c);
}

const char *gb2_last_error(gb2_ctx *c)
{
    if (!c)
        return "no context";
    std::lock_guard<std::mutex> lk(c->err_mu);
    return c->last_error.c_str();
}

static int gb2_batch_upload_impl(gb2_ctx *c, const uint64_t *packed, int64_t n_words, const uint64_t *nmask,
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
    int64_t maxlen = 0, minlen = count > 0 ? INT64_MAX : 0;
    for (int64_t i = 0; i < count; ++i) {
        if (lengths[i] < 0 || offsets[i] < 0 || offsets[i] + words_for(lengths[i]) > n_words)
            return set_err(c, GB2_EINVAL, "sequence %lld lies outside the packed words",
                           (long long)i);
        maxlen = std::max(maxlen, lengths[i]);
        minlen = std::min(minlen, lengths[i]);
    }
    gb2_batch *b = new gb2_batch();
    b->owner = c;
    b->count = count;
    b->n_words = n_words;
    b->max_len = maxlen;
    b->min_len = minlen;
    const size_t wb = (size_t)std::max<int64_t>(n_words, 1) * 8;
    const size_t sb = (size_t)std::max<int64_t>(count, 1) * 8;
    cudaError_t e = dev_alloc(&b->d_packed, wb);
    if (e == cudaSuccess && nmask)
        e = dev_alloc(&b->d_nmask, wb);
    if (e == cudaSuccess)
        e = dev_alloc(&b->d_offsets, sb);
    if (e == cudaSuccess)
        e = dev_alloc(&b->d_lengths, sb);
    auto release = [&]() {
        cudaFree(b->d_packed);
        cudaFree(b->d_nmask);
        cudaFree(b->d_offsets);
        cudaFree(b->d_lengths);
        delete b;
    };
    if (e != cudaSuccess) {
        cudaGetLastError();
        release();
        return set_err(c, GB2_ENOMEM, "device allocation of a %lld-word batch failed",
                       (long long)n_words);
    }
    int rc = GB2_OK;
    if (n_words == 0)
        cudaMemsetAsync(b->d_packed, 0, 8, c->x.st);
    if (!rc)
        rc = h2d(c, b->d_packed, packed, (size_t)n_words * 8, c->x.st);
    if (!rc && nmask)
        rc = h2d(c, b->d_nmask, nmask, (size_t)n_words * 8, c->x.st);
    if (!rc)
        rc = h2d(c, b->d_offsets, offsets, (size_t)count * 8, c->x.st);
    if (!rc)
        rc = h2d(c, b->d_lengths, lengths, (size_t)count * 8, c->x.st);
    if (!rc)
        rc = sync_and_check(c);
    if (rc) {
        release();
        return rc;
    }
    *out = b;
    return GB2_OK;
}

int gb2_batch_upload(gb2_ctx *c, const uint64_t *packed, int64_t n_words, const uint64_t *nmask,
                     const int64_t *offsets, const int64_t *lengths, int64_t count,
                     gb2_batch **out)
{
    return drain_on_error(c, gb2_batch_upload_impl(c, packed, n_words, nmask, offsets, lengths, count, out));
}

int gb2_batch_free(gb2_ctx *c, gb2_batch *b)
{
    if (!c || !b || b->owner != c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->x.st);
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

static int gb2_sw_banded_impl(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_sw_cfg *cfg,
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
    pi.narrow_lengths =
        narrow_range(q->min_len, q->max_len) && narrow_range(r->min_len, r->max_len);
    if (rc)
        return rc;
    if (n == 0)
        return GB2_OK;
    if ((rc = ensure(c, c->out_sw, (size_t)n * sizeof(gb2_sw_result), c->x.st)))
        return rc;
    const int32_t *d_bands = nullptr;
    if (bands) {
        if ((rc = ensure(c, c->bands, (size_t)n * 4, c->x.st)) ||
            (rc = h2d(c, c->bands.p, bands, (size_t)n * 4, c->x.st)))
            return rc;
        d_bands = (const int32_t *)c->bands.p;
    }
    // Large batches run as kResidentParts parts alternating between the two
    // executors, each part's results copied back while the next part computes.
    const int parts = n >= kResidentSplit ? kResidentParts : 1;
    std::vector<int64_t> key{1};
    key_batches(key, q, r);
    key.insert(key.end(), {cfg->match_score, cfg->mismatch, cfg->gap_open, cfg->gap_extend,
                           cfg->band_width, n, flags, bands ? 1 : 0, pi.max_band});
    if (parts == 1) {
        rc = run_graphed(c, c->g_sw, key, flags, nullptr, [&](bool capturing) -> int {
            return sw_core(c, c->x, view_of(q), view_of(r), q->max_len, r->max_len, cfg,
                           d_bands, pi, n, (gb2_sw_result *)c->out_sw.p, flags, !capturing);
        });
        if (rc) {
            cudaStreamSynchronize(c->x.st);
            return rc;
        }
        return d2h_results(c, out, c->out_sw.p, (size_t)n * sizeof(gb2_sw_result));
    }
    const bool out_pinned = is_pinned(out);
    if (!out_pinned && (rc = pin_out(c, (size_t)n * sizeof(gb2_sw_result))))
        return rc;
    gb2_sw_result *const host = out_pinned ? out : (gb2_sw_result *)c->pin_out;
    gb2_sw_result *const dres = (gb2_sw_result *)c->out_sw.p;
    auto issue = [&](bool capturing) -> int {
        CU(c, cudaEventRecord(c->x.ev_fork, c->x.st));  // bands copied before either runs
        CU(c, cudaStreamWaitEvent(c->x2.st, c->x.ev_fork, 0));
        // profiling: one span per call, from the first part's start to the later
        // of the two executors' last kernels (the parts overlap, so their own
        // durations would double-count)
        cudaEvent_t span0 = capturing ? nullptr : prof_begin(c, c->x.st);
        const int64_t per = (n + parts - 1) / parts;
        int r2 = GB2_OK;
        for (int k = 0; k < parts && r2 == GB2_OK; ++k) {
            const int64_t p0 = k * per, m = std::min(per, n - p0);
            Exec &ex = (k & 1) ? c->x2 : c->x;
            SeqView qv = view_of(q), rv = view_of(r);
            qv.offsets += p0;
            qv.lengths += p0;
            rv.offsets += p0;
            rv.lengths += p0;
            r2 = sw_core(c, ex, qv, rv, q->max_len, r->max_len, cfg,
                         d_bands ? d_bands + p0 : nullptr, pi, m, dres + p0, flags, false);
            if (!r2 && !capturing && cudaEventRecord(c->kdone[k], ex.st) != cudaSuccess)
                r2 = set_err(c, GB2_ECUDA, "event record failed");
            if (!r2 && cudaMemcpyAsync(host + p0, dres + p0, (size_t)m * sizeof(gb2_sw_result),
                                       cudaMemcpyDeviceToHost, ex.st) != cudaSuccess)
                r2 = set_err(c, GB2_ECUDA, "result copy failed");
        }
        // the second executor joins the first (a captured graph must end there)
        if (!r2 && (cudaEventRecord(c->ev_join2, c->x2.st) != cudaSuccess ||
                    cudaStreamWaitEvent(c->x.st, c->ev_join2, 0) != cudaSuccess))
            r2 = set_err(c, GB2_ECUDA, "joining the executors failed");
        if (span0 && !r2) {
            cudaStreamWaitEvent(c->st_copy, c->kdone[parts - 2], 0);
            cudaStreamWaitEvent(c->st_copy, c->kdone[parts - 1], 0);
            prof_end(c, span0, c->st_copy);
        } else if (span0) {
            cudaEventDestroy(span0);
        }
        return r2;
    };
    rc = run_graphed(c, c->g_sw, key, flags, (char *)host, issue);
    const cudaError_t e2 = cudaStreamSynchronize(c->x2.st);
    const int rc2 = sync_and_check(c);
    if (rc)
        return rc;
    if (e2 != cudaSuccess)
        return set_err(c, GB2_ECUDA, "second executor: %s", cudaGetErrorString(e2));
    if (rc2)
        return rc2;
    if (!out_pinned)
        memcpy(out, c->pin_out, (size_t)n * sizeof(gb2_sw_result));
    return GB2_OK;
}

int gb2_sw_banded(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_sw_cfg *cfg,
                  const int32_t *bands, int64_t n, gb2_sw_result *out, int flags)
{
    return drain_on_error(c, gb2_sw_banded_impl(c, q, r, cfg, bands, n, out, flags));
}

static int gb2_sw_banded_host_impl(gb2_ctx *c, const uint64_t *q_packed, const int64_t *q_offsets,
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
    SwPlanInfo pi0;
    int rc = sw_validate(c, cfg, nullptr, 0, 0, 0, pi0);  // the config alone
    if (rc || n <= 0)
        return n < 0 ? set_err(c, GB2_EINVAL, "n_pairs < 0") : rc;
    const HostSide hq{q_packed, q_offsets, q_lengths}, hr{r_packed, r_offsets, r_lengths};
    const int nch = (flags >> 16) & 0xff;
    // default: 16 chunks of at least 65,536 pairs (a chunk fills the GPU)
    const int64_t chunk = nch ? std::max<int64_t>(1, (n + nch - 1) / nch)
                              : std::max<int64_t>(1 << 16, (n + 15) / 16);
    return pipeline(c, hq, hr, bands, n, sizeof(gb2_sw_result), out, chunk,
                    [&](Exec &x, SeqView qv, SeqView rv, int64_t qm, int64_t rm, bool narrow,
                        const int32_t *db, const int32_t *hb, int64_t m, void *dout) {
                        SwPlanInfo pi;
                        int r = sw_validate(c, cfg, hb, m, qm, rm, pi);
                        if (r)
                            return r;
                        pi.narrow_lengths = narrow;
                        return sw_core(c, x, qv, rv, qm, rm, cfg, db, pi, m,
                                       (gb2_sw_result *)dout, flags);
                    });
}

int gb2_sw_banded_host(gb2_ctx *c, const uint64_t *q_packed, const int64_t *q_offsets,
                       const int64_t *q_lengths, const uint64_t *r_packed,
                       const int64_t *r_offsets, const int64_t *r_lengths, const gb2_sw_cfg *cfg,
                       const int32_t *bands, int64_t n, gb2_sw_result *out, int flags)
{
    return drain_on_error(c, gb2_sw_banded_host_impl(c, q_packed, q_offsets, q_lengths, r_packed, r_offsets, r_lengths, cfg, bands, n, out, flags));
}

static int gb2_sw_pair_impl(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                int64_t rlen, const gb2_sw_cfg *cfg, gb2_sw_result *out)
{
    if (!c)
        return GB2_EINVAL;
    if (!out || qlen < 0 || rlen < 0 || (qlen > 0 && !q_words) || (rlen > 0 && !r_words))
        return set_err(c, GB2_EINVAL, "bad pair arguments");
    const int64_t qo = 0, ro = 0;
    static const uint64_t zero = 0;
    return gb2_sw_banded_host(c, qlen ? q_words : &zero, &qo, &qlen, rlen ? r_words : &zero, &ro,
                              &rlen, cfg, nullptr, 1, out, GB2_FLAG_PLAIN);
}

int gb2_sw_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                int64_t rlen, const gb2_sw_cfg *cfg, gb2_sw_result *out)
{
    return drain_on_error(c, gb2_sw_pair_impl(c, q_words, qlen, r_words, rlen, cfg, out));
}

static int gb2_wfa_affine_impl(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_wfa_cfg *cfg,
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
    if ((rc = ensure(c, c->out_wfa, (size_t)n * 4, c->x.st)))
        return rc;
    std::vector<int64_t> key{2};
    key_batches(key, q, r);
    key.insert(key.end(), {cfg->x, cfg->o, cfg->e, cfg->max_error, n, flags});
    rc = run_graphed(c, c->g_wfa, key, flags, nullptr, [&](bool) -> int {
        int r2;
        if ((r2 = wfa_begin(c, c->x)))
            return r2;
        return wfa_core(c, c->x, view_of(q), view_of(r), q->max_len, r->max_len, cfg, n,
                        (int32_t *)c->out_wfa.p, flags);
    });
    if (rc) {
        cudaStreamSynchronize(c->x.st);
        return rc;
    }
    if ((rc = wfa_end(c, c->x)))
        return rc;
    return d2h_results(c, out, c->out_wfa.p, (size_t)n * 4);
}

int gb2_wfa_affine(gb2_ctx *c, const gb2_batch *q, const gb2_batch *r, const gb2_wfa_cfg *cfg,
                   int64_t n, int32_t *out, int flags)
{
    return drain_on_error(c, gb2_wfa_affine_impl(c, q, r, cfg, n, out, flags));
}

static int gb2_wfa_affine_host_impl(gb2_ctx *c, const uint64_t *q_packed, const int64_t *q_offsets,
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
    const HostSide hq{q_packed, q_offsets, q_lengths}, hr{r_packed, r_offsets, r_lengths};
    const int nch = (flags >> 16) & 0xff;
    const int64_t chunk = nch ? std::max<int64_t>(1, (n + nch - 1) / nch)
                              : std::max<int64_t>(1024, (n + 3) / 4);
    if ((rc = wfa_begin(c, c->x)) || (rc = wfa_begin(c, c->x2)))
        return rc;
    rc = pipeline(c, hq, hr, nullptr, n, 4, out, chunk,
                  [&](Exec &x, SeqView qv, SeqView rv, int64_t qm, int64_t rm, bool,
                      const int32_t *, const int32_t *, int64_t m, void *dout) {
                      return wfa_core(c, x, qv, rv, qm, rm, cfg, m, (int32_t *)dout, flags);
                  });
    if (rc)
        return rc;
    const int r1 = wfa_end(c, c->x), r2 = wfa_end(c, c->x2);
    return r1 ? r1 : r2;
}

int gb2_wfa_affine_host(gb2_ctx *c, const uint64_t *q_packed, const int64_t *q_offsets,
                        const int64_t *q_lengths, const uint64_t *r_packed,
                        const int64_t *r_offsets, const int64_t *r_lengths,
                        const gb2_wfa_cfg *cfg, int64_t n, int32_t *out, int flags)
{
    return drain_on_error(c, gb2_wfa_affine_host_impl(c, q_packed, q_offsets, q_lengths, r_packed, r_offsets, r_lengths, cfg, n, out, flags));
}

static int gb2_wfa_pair_impl(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                 int64_t rlen, const gb2_wfa_cfg *cfg, int32_t *out)
{
    if (!c)
        return GB2_EINVAL;
    if (!out || qlen < 0 || rlen < 0 || (qlen > 0 && !q_words) || (rlen > 0 && !r_words))
        return set_err(c, GB2_EINVAL, "bad pair arguments");
    const int64_t qo = 0, ro = 0;
    static const uint64_t zero = 0;
    return gb2_wfa_affine_host(c, qlen ? q_words : &zero, &qo, &qlen, rlen ? r_words : &zero, &ro,
                               &rlen, cfg, 1, out, GB2_FLAG_PLAIN);
}

int gb2_wfa_pair(gb2_ctx *c, const uint64_t *q_words, int64_t qlen, const uint64_t *r_words,
                 int64_t rlen, const gb2_wfa_cfg *cfg, int32_t *out)
{
    return drain_on_error(c, gb2_wfa_pair_impl(c, q_words, qlen, r_words, rlen, cfg, out));
}

int gb2_host_alloc(int64_t bytes, void **out)
{
    if (!out || bytes < 0)
        return GB2_EINVAL;
    *out = nullptr;
    if (pinned_alloc(out, (size_t)std::max<int64_t>(bytes, 8)) != cudaSuccess) {
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
    CU(c, cudaEventRecord(c->t0, c->x.st));
    return GB2_OK;
}

int gb2_timer_stop(gb2_ctx *c, float *ms)
{
    if (!c || !ms)
        return GB2_EINVAL;
    cudaSetDevice(c->device);
    CU(c, cudaEventRecord(c->t1, c->x.st));
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
    CU(c, cudaStreamSynchronize(c->x.st));
    harvest_profile(c);
    if (kernel_ms) {
        std::lock_guard<std::mutex> pk(c->prof_mu);
        *kernel_ms = c->kernel_ms;
    }
    if (launches)
        *launches = c->launches.load();
    if (work_units)
        *work_units = c->work_units.load();
    return GB2_OK;
}

// ---- autotuner ---------------------------------------------------------------
int gb2_autotune(gb2_ctx *c, int kind, const gb2_batch *q, const gb2_batch *r, const void *cfgp,
                 const int32_t *bands, int64_t n, int reps, gb2_tune_result *out)
{
    if (!c || !q || !r || !cfgp || !out)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (q->owner != c || r->owner != c)
        return set_err(c, GB2_EINVAL, "batch belongs to another context");
    if (n <= 0 || n > q->count || n > r->count)
        return set_err(c, GB2_EINVAL, "n_pairs must be in [1, batch count]");
    reps = std::max(1, std::min(reps, 50));
    gb2_tune_result res{};
    res.kind = kind;
    std::vector<int> cand;
    int *slot = nullptr;  // the table entry the winner goes to
    size_t out_bytes = 0;
    const void *d_res = nullptr;
    std::function<int(int)> run;  // one run of a candidate on c->x, no host sync
    SwPlanInfo pi;
    int rc;
    if (kind == GB2_TUNE_SW) {
        const gb2_sw_cfg *cfg = (const gb2_sw_cfg *)cfgp;
        res.band_class = classify_band(cfg->band_width);
        switch (res.band_class) {
        case 16: cand = {0, 1}; slot = &c->tune_sw[0]; break;
        case 32: cand = {0, 1, 2}; slot = &c->tune_sw[1]; break;
        case 64: cand = {0, 1}; slot = &c->tune_sw[2]; break;
        case 128: cand = {0, 1}; slot = &c->tune_sw[3]; break;
        default:
            return set_err(c, GB2_EINVAL, "band %d has no kernel variants (16, 32, 64 or 128)",
                           cfg->band_width);
        }
        if ((rc = sw_validate(c, cfg, bands, n, q->max_len, r->max_len, pi)))
            return rc;
        pi.narrow_lengths =
            narrow_range(q->min_len, q->max_len) && narrow_range(r->min_len, r->max_len);
        if (!pi.fast_ok)
            return set_err(c, GB2_EINVAL, "these penalties take the literal kernel (no variants)");
        out_bytes = (size_t)n * sizeof(gb2_sw_result);
        if ((rc = ensure(c, c->out_sw, out_bytes, c->x.st)))
            return rc;
        const int32_t *d_bands = nullptr;
        if (bands) {
            if ((rc = ensure(c, c->bands, (size_t)n * 4, c->x.st)) ||
                (rc = h2d(c, c->bands.p, bands, (size_t)n * 4, c->x.st)))
                return rc;
            d_bands = (const int32_t *)c->bands.p;
        }
        d_res = c->out_sw.p;
        // the candidate goes into the table slot, so with per-pair bands the other
        // classes of the mix run with their installed variants
        run = [=](int v) {
            *slot = v;
            return sw_core(c, c->x, view_of(q), view_of(r), q->max_len, r->max_len, cfg, d_bands,
                           pi, n, (gb2_sw_result *)c->out_sw.p, GB2_FLAG_BATCHED | GB2_FLAG_INT32,
                           false);
        };
    } else if (kind == GB2_TUNE_WFA) {
        const gb2_wfa_cfg *cfg = (const gb2_wfa_cfg *)cfgp;
        if ((rc = wfa_validate(c, cfg, n)))
            return rc;
        // diagonals per thread per round 4, 2, 1 (bits 4-5); blocks per SM (bits 0-3)
        cand = {0x00, 0x04, 0x03, 0x10, 0x20};
        slot = &c->tune_wfa;
        out_bytes = (size_t)n * 4;
        if ((rc = ensure(c, c->out_wfa, out_bytes, c->x.st)))
            return rc;
        d_res = c->out_wfa.p;
        run = [=](int v) {
            int r2;
            if ((r2 = wfa_begin(c, c->x)))
                return r2;
            return wfa_core(c, c->x, view_of(q), view_of(r), q->max_len, r->max_len, cfg, n,
                            (int32_t *)c->out_wfa.p, GB2_FLAG_BATCHED | (v << 8));
        };
    } else {
        return set_err(c, GB2_EINVAL, "kind must be GB2_TUNE_SW or GB2_TUNE_WFA");
    }
    // candidate 0 is the built-in choice, not whatever is installed now
    const int saved = *slot;
    *slot = 0;
    auto finish = [&](int status) {
        if (status != GB2_OK)
            *slot = saved;
        cudaStreamSynchronize(c->x.st);
        return status;
    };
    auto settle = [&]() -> int {  // wait for the run; WFA reports its error flag
        if (kind == GB2_TUNE_WFA)
            return wfa_end(c, c->x);
        CU(c, cudaStreamSynchronize(c->x.st));
        return GB2_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return finish(set_err(c, GB2_ECUDA, "creating timing events failed"));
    }
    std::vector<char> first(out_bytes), cur(out_bytes);
    int best = cand[0];
    float best_ms = 0.f;
    rc = GB2_OK;
    for (size_t i = 0; i < cand.size() && rc == GB2_OK; ++i) {
        const int v = cand[i];
        if ((rc = run(v)) || (rc = settle()))
            break;
        // results of every candidate equal the first's
        if (cudaMemcpy(i ? cur.data() : first.data(), d_res, out_bytes, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
            rc = set_err(c, GB2_ECUDA, "reading back the results failed");
            break;
        }
        if (i && memcmp(first.data(), cur.data(), out_bytes) != 0) {
            rc = set_err(c, GB2_EKERNEL, "variant %#x gives other results than variant %#x", v,
                         cand[0]);
            break;
        }
        std::vector<float> t;
        for (int k = 0; k < reps && rc == GB2_OK; ++k) {
            float ms = 0.f;
            if (cudaEventRecord(e0, c->x.st) != cudaSuccess || (rc = run(v)) ||
                cudaEventRecord(e1, c->x.st) != cudaSuccess || (rc = settle()) ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                if (rc == GB2_OK)
                    rc = set_err(c, GB2_ECUDA, "timing a variant failed");
                break;
            }
            t.push_back(ms);
        }
        if (rc)
            break;
        std::sort(t.begin(), t.end());
        const float med = t[t.size() / 2];
        res.variant[res.n_candidates] = v;
        res.ms[res.n_candidates] = med;
        ++res.n_candidates;
        if (i == 0 || med < best_ms) {
            best = v;
            best_ms = med;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return finish(rc);
    *slot = best;
    res.chosen = best;
    *out = res;
    return finish(GB2_OK);
}

int gb2_tune_set(gb2_ctx *c, int kind, int band_class, int variant)
{
    if (!c || variant < 0 || variant > 0xff)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (kind == GB2_TUNE_WFA) {
        c->tune_wfa = variant;
        return GB2_OK;
    }
    const int slot = band_class == 16 ? 0 : band_class == 32 ? 1 : band_class == 64 ? 2
                   : band_class == 128 ? 3 : -1;
    if (kind != GB2_TUNE_SW || slot < 0)
        return set_err(c, GB2_EINVAL, "no tuning entry for kind %d, band class %d", kind,
                       band_class);
    c->tune_sw[slot] = variant;
    return GB2_OK;
}

int gb2_tune_get(gb2_ctx *c, int kind, int band_class, int *variant)
{
    if (!c || !variant)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (kind == GB2_TUNE_WFA) {
        *variant = c->tune_wfa;
        return GB2_OK;
    }
    const int slot = band_class == 16 ? 0 : band_class == 32 ? 1 : band_class == 64 ? 2
                   : band_class == 128 ? 3 : -1;
    if (kind != GB2_TUNE_SW || slot < 0)
        return set_err(c, GB2_EINVAL, "no tuning entry for kind %d, band class %d", kind,
                       band_class);
    *variant = c->tune_sw[slot];
    return GB2_OK;
}

int gb2_stats_reset(gb2_ctx *c)
{
    if (!c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    CU(c, cudaStreamSynchronize(c->x.st));
    harvest_profile(c);
    {
        std::lock_guard<std::mutex> pk(c->prof_mu);
        c->kernel_ms = 0;
    }
    c->launches = 0;
    c->work_units = 0;
    return GB2_OK;
}

int gb2_set_profiling(gb2_ctx *c, int enable)
{
    if (!c)
        return GB2_EINVAL;
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
    const int rc = ensure(c, c->flush, bytes, c->x.st);
    if (rc)
        return rc;
    CU(c, cudaMemsetAsync(c->flush.p, (int)(c->launches.load() & 0xff), bytes, c->x.st));
    return GB2_OK;
}

int gb2_int_peak(gb2_ctx *c, int kind, double *gops)
{
    if (!c || !gops || kind < 0 || kind > 12)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const int rc = ensure(c, c->x.work, 64, c->x.st);
    if (rc)
        return rc;
    CU(c, cudaMemsetAsync(c->x.work.p, 0, 64, c->x.st));
    const int block = 256, grid = c->sm_count * 8, iters = 4096;
    CU(c, launch_int_peak(kind, grid, block, 64, (uint32_t *)c->x.work.p, c->x.st));
    CU(c, cudaEventRecord(c->t0, c->x.st));
    CU(c, launch_int_peak(kind, grid, block, iters, (uint32_t *)c->x.work.p, c->x.st));
    CU(c, cudaEventRecord(c->t1, c->x.st));
    CU(c, cudaEventSynchronize(c->t1));
    float ms = 0.f;
    CU(c, cudaEventElapsedTime(&ms, c->t0, c->t1));
    const double ops = (double)grid * block * iters * 8.0;
    *gops = ops / (ms * 1e-3) / 1e9;
    return GB2_OK;
}

}  // extern "C"
