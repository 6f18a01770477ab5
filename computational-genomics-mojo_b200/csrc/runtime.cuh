// runtime.cuh -- host runtime types shared by api.cu and server.cu (not installed).
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <mutex>
#include <string>
#include <vector>

#include "gb2_internal.cuh"

namespace gb2 {

constexpr int kAux = 4;            // auxiliary streams for concurrent band classes
// 16, 32, 64, 128 (int32 registers), literal, packed 16, packed 32 (narrow keys),
// packed 16, 32, 64, 128 (wide keys)
constexpr int kSwClasses = 11;
constexpr int kLenBuckets = 1024;  // length buckets per class
constexpr int64_t kSwSmallBatch = 16384;  // SW batches this small take the widest lane split
constexpr int64_t kInlineScanPairs = 8192;  // host batches this small are scanned inline
constexpr int64_t kPinChunk = 32ll << 20;
// Packed int16x2 kernels: every cell they compute (the in-matrix ones, and the
// row past the query end, which adds at most `match`) stays below these, checked
// as match * (min(qlen, rlen) + 1): H*128 + column fits 16 bits (narrow keys),
// H*8 + 7 fits a signed 16-bit half (wide keys).
constexpr int64_t kPackHmax = 511;
constexpr int64_t kWideHmax = 4094;
constexpr int64_t kWfaScratchCap = 8ll << 30;  // WFA rings of all warps, bytes
constexpr int64_t kWfaTeamMinLen = 2048;       // shortest WFA pair aligned by a whole block
constexpr int64_t kTierDumpCap = 1ll << 30;    // bytes of suspended-pair records per transition
// WFA bound pass: batches whose longest sequence has at least kWfaBoundMinLen
// bases run it, over a band of +-kWfaBoundBand diagonals
constexpr int64_t kWfaBoundMinLen = 1024;
// WFA: batches of fewer pairs per SM than this skip the two-warp tier
constexpr int64_t kWfaTwoWarpMinPairsPerSm = 160;
constexpr int32_t kWfaBoundBand = 64;

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    // set: grow by stream-ordered free and allocation from this pool, with
    // headroom, so growing never synchronises the device (the server's slots)
    cudaMemPool_t pool = nullptr;
};

// An executor: one stream (plus auxiliary streams for concurrent band
// classes) and the planning / scratch buffers its launches use.  Work on one
// executor is ordered; separate executors can overlap on the device.
struct Exec {
    cudaStream_t st = nullptr;
    cudaStream_t aux[kAux] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kAux] = {};
    DevBuf keys, queue, counts, seg, counters, scratch64, scratch32, work, errflag;
    DevBuf tierq, dumps;  // tiered WFA: the M/L/G queues and the suspended pairs' records
    DevBuf ubound;        // WFA: per pair, the bound pass's cost (an upper bound of the optimum)
};

// Device buffers of the WFA CIGAR entry point (grow-only, per context).
struct CigarBufs {
    DevBuf cost, hist, pairs, arena_off, arena, runs, run_off, run_count, out_off, out;
};
// WFA history arena, bytes at most (and at most half the free device memory):
// 38 GB of history for 20,000 long pairs then runs as one group, not three
// (137k -> 170-178k pairs/s)
constexpr int64_t kCigarArenaCap = 64ll << 30;

// One set of device buffers of the end-to-end pipeline.
struct PipeSet {
    DevBuf qw, rw, qo, ql, ro, rl, bands, out, len32;
    // copied: inputs on the device; ready: offsets rebuilt (contiguous chunks);
    // kern: the chunk's kernels ended; done: its results are back on the host
    cudaEvent_t copied = nullptr, ready = nullptr, kern = nullptr, done = nullptr;
};
constexpr int kPipeSets = 6;  // chunks in flight in the host pipeline
constexpr int64_t kResidentSplit = 1 << 18;  // resident SW batches this large run in parts
constexpr int kResidentParts = 4;

// Replay cache of one resident entry point (gb2_sw_banded, gb2_wfa_affine),
// used with GB2_FLAG_GRAPH.  The device work of a call is captured into a CUDA graph on the second call in
// a row with the same key -- everything the host decides the launches from:
// the batches' device arrays and sizes, the scoring, n_pairs, flags -- and
// while the context's buffers keep their addresses (gen), later calls with
// that key launch the graph instead of re-issuing memsets, planning kernels,
// the alignment kernels and the stream forks and joins one by one.  Result
// copies to the caller's host array are memcpy nodes whose destination is
// updated when the array moves.  Calls made while profiling is on run eagerly.
struct GraphCache {
    std::vector<int64_t> key;
    uint64_t gen = 0;
    bool failed = false;           // capture failed for this key: stay eager
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;           // kernel nodes, for the launch statistics
    struct Copy {
        cudaGraphNode_t node;
        size_t dst_off, bytes;     // destination offset from the call's host base
        const void *src;
    };
    std::vector<Copy> copies;
    char *host = nullptr;          // host base the copy nodes currently hold
    void reset()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        key.clear();
        copies.clear();
        kernels = 0;
        host = nullptr;
        failed = false;
    }
};

struct SwPlanInfo {
    bool fast_ok;       // the register kernels apply (sign conditions on the scores)
    bool pack_ok;       // the packed int16x2 kernel applies (scores also small)
    bool wide_ok;       // ... and with its wide keys (match <= 127)
    int32_t max_band;
    bool uniform_band;  // no per-pair bands
    // set by the caller when every pair's lengths lie in a narrow range: a
    // length-sorted queue would order nothing, so the batched path skips it
    bool narrow_lengths = false;
};

// Lengths [lo, hi] count as narrow when hi is within 1/8 (at least 16 bases)
// of lo.
inline bool narrow_range(int64_t lo, int64_t hi)
{
    return hi - lo <= std::max<int64_t>(16, lo / 8);
}

}  // namespace gb2

struct gb2_batch {
    uint64_t *d_packed = nullptr;
    uint64_t *d_nmask = nullptr;
    int64_t *d_offsets = nullptr;
    int64_t *d_lengths = nullptr;
    int64_t count = 0, n_words = 0, max_len = 0, min_len = 0;
    gb2_ctx *owner = nullptr;
};

struct gb2_ctx {
    int device = 0;
    int sm_count = 148;
    gb2::Exec x;                  // the executor of the blocking entry points
    gb2::Exec x2;                 // second executor: the host pipeline alternates chunks
    cudaStream_t st_copy = nullptr;
    cudaStream_t st_prep = nullptr;  // host pipeline: offset rebuild of contiguous chunks
    cudaStream_t st_back = nullptr;  // host pipeline: result copies to the host
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::mutex mu;                // serialises the entry points of this context
    std::mutex err_mu;
    std::string last_error;
    gb2::DevBuf out_sw, out_wfa, bands, flush;
    void *pin[2] = {nullptr, nullptr};  // pinned staging halves for pageable uploads
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
    std::mutex pin_mu;
    void *pin_out = nullptr;
    size_t pin_out_cap = 0;
    void *pin_len32 = nullptr;  // int32 lengths of contiguous chunks (host pipeline)
    size_t pin_len32_cap = 0;
    gb2::PipeSet pipe[gb2::kPipeSets];
    gb2::CigarBufs cig;
    cudaEvent_t kdone[gb2::kResidentParts] = {};  // last kernel of each resident part
    cudaEvent_t ev_join2 = nullptr;  // second executor joined back into the first
    uint64_t buf_gen = 0;            // bumped whenever a context buffer is reallocated
    gb2::GraphCache g_sw, g_wfa;     // replay caches of gb2_sw_banded / gb2_wfa_affine
    // variants installed by gb2_autotune / gb2_tune_set (0 = built-in choice):
    // SW register kernels of bands 16, 32, 64, 128; the 4-warp WFA kernel
    int tune_sw[4] = {0, 0, 0, 0};
    int tune_wfa = 0;
    // statistics
    std::atomic<bool> profiling{false};
    std::mutex prof_mu;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_pending;
    double kernel_ms = 0.0;
    std::atomic<int64_t> launches{0};
    std::atomic<int64_t> work_units{0};
};

namespace gb2 {

int set_err(gb2_ctx *c, int code, const char *fmt, ...);

// Allocation fault injection (gb2_debug_fail_alloc): a countdown per kind;
// the allocation that finds it at zero fails as out of memory, and the
// countdown turns off (-1).  Every device and pinned allocation of the
// library goes through these helpers.
extern std::atomic<int64_t> g_fail_dev, g_fail_pin;
inline bool injected_failure(std::atomic<int64_t> &cd)
{
    int64_t v = cd.load();
    while (v >= 0) {
        if (cd.compare_exchange_weak(v, v - 1))
            return v == 0;
    }
    return false;
}
template <typename T>
inline cudaError_t dev_alloc(T **p, size_t bytes)
{
    if (injected_failure(g_fail_dev))
        return cudaErrorMemoryAllocation;
    return cudaMalloc(reinterpret_cast<void **>(p), bytes);
}
template <typename T>
inline cudaError_t dev_alloc_pool(T **p, size_t bytes, cudaMemPool_t pool, cudaStream_t st)
{
    if (injected_failure(g_fail_dev))
        return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, st);
}
template <typename T>
inline cudaError_t pinned_alloc(T **p, size_t bytes)
{
    if (injected_failure(g_fail_pin))
        return cudaErrorMemoryAllocation;
    return cudaMallocHost(reinterpret_cast<void **>(p), bytes);
}

#define GB2_CU(ctx, call)                                                                  \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return ::gb2::set_err((ctx),                                                   \
                                  e_ == cudaErrorMemoryAllocation ? GB2_ENOMEM : GB2_ECUDA, \
                                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                                  __LINE__);                                               \
    } while (0)

// Returns rc; when rc is an error, first waits for every stream of the
// context, so a failed call leaves no work of its own in flight.
int drain_on_error(gb2_ctx *c, int rc);

int exec_init(Exec &x);
void exec_free(Exec &x);
// Grows b to at least `bytes`; an existing buffer is freed after `st` drains.
int ensure(gb2_ctx *c, DevBuf &b, size_t bytes, cudaStream_t st);
bool is_pinned(const void *p);
// Host-to-device copy on st: pinned sources by DMA, pageable ones through the
// context's two pinned staging halves.
int h2d(gb2_ctx *c, void *dst, const void *src, size_t bytes, cudaStream_t st);
int64_t words_for(int64_t len);
void harvest_profile(gb2_ctx *c);

int sw_validate(gb2_ctx *c, const gb2_sw_cfg *cfg, const int32_t *bands, int64_t n, int64_t qmax,
                int64_t rmax, SwPlanInfo &pi);
// Enqueues Smith-Waterman for n pairs of (qv, rv) on executor x; results to d_out.
// profile: record the launches' duration when the context is profiling.
int sw_core(gb2_ctx *c, Exec &x, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
            const gb2_sw_cfg *cfg, const int32_t *d_bands, const SwPlanInfo &pi, int64_t n,
            gb2_sw_result *d_out, int flags, bool profile = true);
int wfa_validate(gb2_ctx *c, const gb2_wfa_cfg *cfg, int64_t n);
// Clears the WFA error flag and work counter of x (once per call, before the
// first wfa_core of that call).
int wfa_begin(gb2_ctx *c, Exec &x);
// d_hist (optional): per pair, the history cell bytes the CIGAR pass needs.
int wfa_core(gb2_ctx *c, Exec &x, SeqView qv, SeqView rv, int64_t qmax, int64_t rmax,
             const gb2_wfa_cfg *cfg, int64_t n, int32_t *d_out, int flags,
             int64_t *d_hist = nullptr);
// Reads back x's WFA error flag and work counter (synchronises x's stream),
// folds the work into the context's statistics and turns the flag into a status.
int wfa_end(gb2_ctx *c, Exec &x);

}  // namespace gb2
