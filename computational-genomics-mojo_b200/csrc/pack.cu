// pack.cu -- device-side SequenceBatch construction from ASCII.
//
// gb2_batch_from_ascii performs SequenceBatch.add_sequence
// (genomics/core/sequence.mojo:38-66) for a whole batch on the GPU: ACGT /
// acgt become 2-bit codes packed MSB-first, 32 per word
// (genomics/core/dna.mojo:25-40, :96-100); any other byte is stored as A and
// flagged in the word's NMask, bit i = position i (dna.mojo:107-141); tail
// bits of a sequence's last word are zero.  Sequences are laid out in input
// order, each starting at the word after the previous one ends, as
// add_sequence appends them.
//
// One warp per sequence; each lane builds whole words.  The kernel is bound
// by HBM: one byte read and a quarter byte of packed word plus a quarter byte
// of NMask written per base.
#include <algorithm>

#include "runtime.cuh"

using namespace gb2;

namespace {

__device__ __forceinline__ uint32_t code_of(uint32_t ch, uint32_t &is_n)
{
    switch (ch) {
    case 'A': case 'a': is_n = 0; return 0;
    case 'C': case 'c': is_n = 0; return 1;
    case 'G': case 'g': is_n = 0; return 2;
    case 'T': case 't': is_n = 0; return 3;
    default: is_n = 1; return 0;
    }
}

__global__ void __launch_bounds__(256)
k_pack_ascii(const uint8_t *__restrict__ ascii, const int64_t *__restrict__ starts,
             const int64_t *__restrict__ lengths, const int64_t *__restrict__ word_offsets,
             int64_t count, uint64_t *__restrict__ packed, uint64_t *__restrict__ nmask)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < count; s += nwarps) {
        const int64_t len = lengths[s];
        const uint8_t *src = ascii + starts[s];
        const int64_t w0 = word_offsets[s];
        const int64_t nw = (len + 31) >> 5;
        for (int64_t w = lane; w < nw; w += 32) {
            const int64_t b0 = w << 5;
            const int n = (int)min((int64_t)32, len - b0);
            uint64_t word = 0, nm = 0;
            for (int i = 0; i < n; ++i) {
                uint32_t isn;
                const uint32_t c = code_of(__ldg(src + b0 + i), isn);
                word |= (uint64_t)c << (62 - 2 * i);
                nm |= (uint64_t)isn << i;
            }
            packed[w0 + w] = word;
            nmask[w0 + w] = nm;
        }
    }
}

}  // namespace

extern "C" {

static int gb2_batch_from_ascii_impl(gb2_ctx *c, const uint8_t *ascii, int64_t ascii_bytes,
                         const int64_t *starts, const int64_t *lengths, int64_t count,
                         gb2_batch **out)
{
    if (!c || !out)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    *out = nullptr;
    if (count < 0 || ascii_bytes < 0 || (count > 0 && (!starts || !lengths)) ||
        (ascii_bytes > 0 && !ascii))
        return set_err(c, GB2_EINVAL, "ascii batch arrays missing or sizes negative");
    std::vector<int64_t> woff((size_t)std::max<int64_t>(count, 1));
    int64_t words = 0, maxlen = 0, minlen = count > 0 ? INT64_MAX : 0;
    for (int64_t i = 0; i < count; ++i) {
        if (lengths[i] < 0 || starts[i] < 0 || starts[i] + lengths[i] > ascii_bytes)
            return set_err(c, GB2_EINVAL, "sequence %lld lies outside the ascii buffer",
                           (long long)i);
        woff[(size_t)i] = words;
        words += words_for(lengths[i]);
        maxlen = std::max(maxlen, lengths[i]);
        minlen = std::min(minlen, lengths[i]);
    }
    gb2_batch *b = new gb2_batch();
    b->owner = c;
    b->count = count;
    b->n_words = words;
    b->max_len = maxlen;
    b->min_len = minlen;
    uint8_t *d_ascii = nullptr;
    int64_t *d_starts = nullptr;
    const size_t wb = (size_t)std::max<int64_t>(words, 1) * 8;
    const size_t sb = (size_t)std::max<int64_t>(count, 1) * 8;
    cudaError_t e = dev_alloc(&b->d_packed, wb);
    if (e == cudaSuccess)
        e = dev_alloc(&b->d_nmask, wb);
    if (e == cudaSuccess)
        e = dev_alloc(&b->d_offsets, sb);
    if (e == cudaSuccess)
        e = dev_alloc(&b->d_lengths, sb);
    if (e == cudaSuccess)
        e = dev_alloc(&d_ascii, (size_t)std::max<int64_t>(ascii_bytes, 1));
    if (e == cudaSuccess)
        e = dev_alloc(&d_starts, sb);
    int rc = GB2_OK;
    if (e != cudaSuccess) {
        cudaGetLastError();
        rc = set_err(c, GB2_ENOMEM, "device allocation for %lld ascii bytes failed",
                     (long long)ascii_bytes);
    }
    Exec &x = c->x;
    if (!rc)
        rc = h2d(c, d_ascii, ascii, (size_t)ascii_bytes, x.st);
    if (!rc)
        rc = h2d(c, d_starts, starts, (size_t)count * 8, x.st);
    if (!rc)
        rc = h2d(c, b->d_lengths, lengths, (size_t)count * 8, x.st);
    if (!rc)
        rc = h2d(c, b->d_offsets, woff.data(), (size_t)count * 8, x.st);
    if (!rc && count > 0) {
        const int64_t blocks = std::min<int64_t>((count + 7) / 8, (int64_t)c->sm_count * 64);
        k_pack_ascii<<<(int)blocks, 256, 0, x.st>>>(d_ascii, d_starts, b->d_lengths, b->d_offsets,
                                                     count, b->d_packed, b->d_nmask);
        if (cudaGetLastError() != cudaSuccess)
            rc = set_err(c, GB2_ECUDA, "pack kernel launch failed");
        c->launches += 1;
    }
    if (!rc && words == 0) {
        cudaMemsetAsync(b->d_packed, 0, 8, x.st);
        cudaMemsetAsync(b->d_nmask, 0, 8, x.st);
    }
    if (!rc && cudaStreamSynchronize(x.st) != cudaSuccess)
        rc = set_err(c, GB2_ECUDA, "pack kernel failed");
    cudaFree(d_ascii);
    cudaFree(d_starts);
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

int gb2_batch_from_ascii(gb2_ctx *c, const uint8_t *ascii, int64_t ascii_bytes,
                         const int64_t *starts, const int64_t *lengths, int64_t count,
                         gb2_batch **out)
{
    return drain_on_error(c, gb2_batch_from_ascii_impl(c, ascii, ascii_bytes, starts, lengths, count, out));
}

int gb2_batch_download(gb2_ctx *c, const gb2_batch *b, uint64_t *packed, uint64_t *nmask,
                       int64_t *offsets, int64_t *lengths)
{
    if (!c || !b || b->owner != c)
        return GB2_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    Exec &x = c->x;
    if (packed && b->n_words)
        GB2_CU(c, cudaMemcpyAsync(packed, b->d_packed, (size_t)b->n_words * 8,
                                  cudaMemcpyDeviceToHost, x.st));
    if (nmask && b->n_words) {
        if (!b->d_nmask)
            return set_err(c, GB2_EINVAL, "batch was uploaded without NMask words");
        GB2_CU(c, cudaMemcpyAsync(nmask, b->d_nmask, (size_t)b->n_words * 8,
                                  cudaMemcpyDeviceToHost, x.st));
    }
    if (offsets && b->count)
        GB2_CU(c, cudaMemcpyAsync(offsets, b->d_offsets, (size_t)b->count * 8,
                                  cudaMemcpyDeviceToHost, x.st));
    if (lengths && b->count)
        GB2_CU(c, cudaMemcpyAsync(lengths, b->d_lengths, (size_t)b->count * 8,
                                  cudaMemcpyDeviceToHost, x.st));
    GB2_CU(c, cudaStreamSynchronize(x.st));
    return GB2_OK;
}

}  // extern "C"
