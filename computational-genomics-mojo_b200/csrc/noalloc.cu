// noalloc.cu -- gb2_wfa_affine_noalloc: gap-affine WFA costs with no device
// allocation at all.
//
// Who needs it: callers whose device memory belongs to someone else -- a
// host runtime or framework that has reserved the GPU's memory for its own
// allocator, a plug-in that must live inside a fixed memory budget -- and
// request loops that may not allocate (or risk an allocation failure) while
// serving.  They pass inputs and outputs that they already own; the
// wavefront scratch comes from the fixed array below instead of cudaMalloc.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds GB2_NOALLOC_SCRATCH_BYTES of it until the process exits.
// Host code cannot use the symbol itself as a device address (in host code
// it names a host-side stand-in); the first call on each device looks up the
// real address with cudaGetSymbolAddress while that device is current and
// caches it.  That first call should come before any stream capture.
//
// All calls share the array and it keeps the previous call's contents: the
// header words (error flag, queue counter) are cleared at the start of every
// call, and the kernel initialises every ring position before reading it.
// Two calls that overlap on the GPU (different host threads, or different
// streams) race on the array; callers must serialise them.
#include <mutex>

#include "gb2_internal.cuh"

namespace {

constexpr int64_t kHeaderBytes = 256;  // [0] error flag, [16] queue counter

static __device__ __align__(256) unsigned char g_noalloc_scratch[GB2_NOALLOC_SCRATCH_BYTES];

std::mutex g_addr_mu;
constexpr int kMaxDevices = 64;
void *g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device, with that device current).
int scratch_address(void **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ECUDA;
    }
    if (dev < 0 || dev >= kMaxDevices)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return GB2_ECUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return GB2_OK;
}

int gcd_i(int a, int b)
{
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

extern "C" int gb2_wfa_affine_noalloc(const uint64_t *q_packed, int64_t q_words,
                                      const int64_t *q_offsets, const int64_t *q_lengths,
                                      const uint64_t *r_packed, int64_t r_words,
                                      const int64_t *r_offsets, const int64_t *r_lengths,
                                      int64_t max_qlen, int64_t max_rlen, const gb2_wfa_cfg *cfg,
                                      int64_t n_pairs, int32_t *out_cost, void *stream)
{
    if (!cfg || n_pairs < 0 || max_qlen < 0 || max_rlen < 0)
        return GB2_EINVAL;
    if (cfg->x < 1 || cfg->e < 1 || cfg->o < 0 || cfg->max_error < 0)
        return GB2_EINVAL;
    const int g = gcd_i(cfg->x, gcd_i(cfg->o, cfg->e));
    const int hm = (cfg->x / g > (cfg->o + cfg->e) / g ? cfg->x / g : (cfg->o + cfg->e) / g) + 1;
    const int hie = cfg->e / g + 1;
    if (hm > 32 || hie > 32)
        return GB2_EINVAL;
    if (n_pairs == 0)
        return GB2_OK;
    if (!q_packed || !q_offsets || !q_lengths || !r_packed || !r_offsets || !r_lengths ||
        !out_cost || q_words < 1 || r_words < 1)
        return GB2_EINVAL;
    if (max_qlen >= (1ll << 30) || max_rlen >= (1ll << 30))
        return GB2_ESCRATCH;

    // One warp per pair in flight; each warp needs its ring slots.  The
    // kernel runs 4 warps per block, so at least one block must fit.
    const int nslot = hm + 2 * hie;
    const int64_t slot_width = ((max_qlen + max_rlen + 5) + 31) & ~int64_t(31);
    const int64_t per_warp = (int64_t)nslot * slot_width * (int64_t)sizeof(int32_t);
    const int64_t fit_warps = (GB2_NOALLOC_SCRATCH_BYTES - kHeaderBytes) / per_warp;
    if (fit_warps < 4)
        return GB2_ESCRATCH;

    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc)
        return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ECUDA;
    }
    int64_t blocks = fit_warps / 4;
    const int64_t want = (n_pairs + 3) / 4;
    if (blocks > want)
        blocks = want;
    // as many blocks as stay resident (the allocating path's grid), at most
    const int64_t resident = (int64_t)sms * gb2::wfa_blocks_per_sm(0, 4);
    if (blocks > resident)
        blocks = resident;

    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *const hdr = (unsigned char *)base;
    int *const err_flag = (int *)hdr;
    int *const counter = (int *)(hdr + 16);
    int32_t *const rings = (int32_t *)(hdr + kHeaderBytes);
    if (cudaMemsetAsync(hdr, 0, kHeaderBytes, st) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ECUDA;
    }
    gb2::SeqView qv{q_packed, q_offsets, q_lengths, 0, q_words};
    gb2::SeqView rv{r_packed, r_offsets, r_lengths, 0, r_words};
    gb2::WfaParams p{cfg->x, cfg->o, cfg->e, cfg->max_error};
    const gb2::PairList none{nullptr, 0, nullptr, counter};
    const gb2::PairList pl{nullptr, n_pairs, nullptr, counter};
    if (gb2::launch_wfa(0, 4, qv, rv, p, none, pl, out_cost, rings, slot_width, (int)blocks,
                        err_flag, nullptr, nullptr, st) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ECUDA;
    }
    int flag = 0;
    if (cudaMemcpyAsync(&flag, err_flag, sizeof flag, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return GB2_ECUDA;
    }
    // the flag means a pair was longer than max_qlen/max_rlen said (its cost is -2)
    return flag ? GB2_EINVAL : GB2_OK;
}
