// gb2_internal.cuh -- shared declarations of libgenomics_b200 (not installed).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "genomics_b200.h"

namespace gb2 {

// Device view of one SequenceBatch side of a pair list.
struct SeqView {
    const uint64_t *packed;  // packed words resident on the device
    const int64_t *offsets;  // word offset of each sequence (SequenceBatch.offsets)
    const int64_t *lengths;  // bases of each sequence (SequenceBatch.lengths)
    int64_t word_base;       // offsets[i] - word_base indexes `packed`
    int64_t n_words;         // words in `packed` (reads are clamped to it)
};

// Which pairs a launch processes: queue[start .. start+n) of pair indices
// (queue == nullptr: pairs [0, n)).  When seg != nullptr the device array
// seg[0..1] = [start, end) overrides n (set by the bucketing kernels).
// counter != nullptr hands out queue slots dynamically (atomics); it must
// be zero at launch.
struct PairList {
    const int32_t *queue;
    int64_t n;
    const int64_t *seg;
    int *counter;
};

// Loads the 64-bit window of 32 bases starting at base `pos` of a sequence
// whose first word is `word0` (global word index); words outside
// [0, n_words) read as the nearest valid word, so any pos is safe to load
// (callers mask or ignore bases outside the sequence).
__device__ __forceinline__ uint64_t load_window64(const uint64_t *__restrict__ packed,
                                                  int64_t n_words, int64_t word0,
                                                  int64_t pos)
{
    int64_t w = word0 + (pos >> 5);
    int sh = (int)(pos & 31) * 2;
    int64_t w0 = w < 0 ? 0 : (w >= n_words ? n_words - 1 : w);
    int64_t w1 = w + 1 < 0 ? 0 : (w + 1 >= n_words ? n_words - 1 : w + 1);
    uint64_t a = __ldg(packed + w0);
    uint64_t b = __ldg(packed + w1);
    return sh ? ((a << sh) | (b >> (64 - sh))) : a;
}

// Base at position pos (MSB-first), genomics/core/dna.mojo:96-100.
// Resolves a PairList on the device: returns the queue base and sets n.
__device__ __forceinline__ const int32_t *pairs_resolve(const PairList &pl, int64_t &n)
{
    if (pl.seg) {
        const int64_t s0 = pl.seg[0];
        n = pl.seg[1] - s0;
        return pl.queue + s0;
    }
    n = pl.n;
    return pl.queue;
}

}  // namespace gb2

// Launch helpers implemented in the kernel translation units.
namespace gb2 {

struct SwParams {
    int32_t match, mismatch, go, ge;
};

// band_class flags selecting the packed int16x2 kernel: kPack16 with keys for
// scores up to 511 (bands 16 and 32), kPackWide with group keys for scores up
// to 4094 (bands 16, 32, 64, 128).
constexpr int kPack16 = 0x100;
constexpr int kPackWide = 0x200;

// Smith-Waterman launch over a list of pair indices (queue == nullptr means
// pairs [0, n)).  `bands` (device, may be nullptr) overrides `band`.
// band_class: 16, 32, 64, 128 for the register kernels, 0 for the literal
// per-pair kernel.  Returns a cudaError_t.
cudaError_t launch_sw(int band_class, int variant, SeqView q, SeqView r, SwParams p,
                      int32_t band, const int32_t *bands, PairList pl, gb2_sw_result *out,
                      int64_t *scratch, int64_t scratch_stride, int grid, cudaStream_t st);

// The naive baseline: one 128-thread block per pair, pairs in input order
// (grid = n), int32 band rows in shared memory (2 * (2 * max_band + 1) ints).
constexpr int32_t kSwNaiveMaxBand = 4096;
cudaError_t launch_sw_naive(SeqView q, SeqView r, SwParams p, int32_t band, const int32_t *bands,
                            int32_t max_band, int64_t n, gb2_sw_result *out, cudaStream_t st);

// Pairs per 128-thread block, and resident blocks per SM, of a kernel variant.
int sw_pairs_per_block(int band_class, int variant);
int sw_blocks_per_sm(int band_class, int variant);

struct WfaParams {
    int32_t x, o, e, max_error;
};

// WFA over two pair lists: `longs` one pair per block of block_warps warps
// (4, or kWfaWideWarps for the wide kernel), then `shorts` one pair per warp.
// scratch: grid * block_warps regions of nslot * slot_width int32.
constexpr int kWfaWideWarps = 16;
// Resident blocks per SM of the WFA kernel variant.
int wfa_blocks_per_sm(int variant, int block_warps);
// hist (optional): per pair, the bytes of the cell part of its WFA history
// record (wfa_hist_cell_bytes summed over the visited scores), 0 when the
// cost is -1.
cudaError_t launch_wfa(int variant, int block_warps, SeqView q, SeqView r, WfaParams p,
                       PairList longs, PairList shorts, int32_t *out, int32_t *scratch,
                       int64_t slot_width, int grid, int *err_flag, int64_t *work, int64_t *hist,
                       cudaStream_t st);

// Tiered WFA (wfa_tiers.cu): tiers 0..4 align a pair with 1, 2, 4, 8 and 16
// warps, rings of W int16 per slot in shared memory; tier kWfaShared (G)
// sixteen warps, int32 rings in global memory covering every diagonal.
constexpr int kWfaShared = 5;  // tiers with their rings in shared memory
struct WfaTierPlan {
    int nslot;
    int32_t W[kWfaShared + 1], H[kWfaShared + 1];  // window per slot row; element of diagonal 0
    int32_t seq_cap[kWfaShared + 1];     // 16-base window entries of a sequence copy
    int64_t team_bytes[kWfaShared + 1];  // shared bytes per team
    int64_t ring_bytes[kWfaShared + 1];  // of them, the ring
    int64_t dump_stride[kWfaShared];     // bytes of a suspended pair's record, per source tier
    bool usable[kWfaShared + 1];         // the window holds at least 64 diagonals
    int64_t gring_block_bytes; // G tier ring region of one block
};
WfaTierPlan wfa_tier_plan(const WfaParams &p, int64_t qmax, int64_t rmax);

// Inputs and outputs of one tier launch.  Input: list (int32 pair indices,
// nullptr = 0..n-1) or ents ({pair, dump record or -1}); n, or *n_dev when set,
// or seg[0..1] = [start, end) of list; ctr hands items out (zeroed).  Output:
// suspended pairs go to next (count next_n) with their record in dumps_out
// (dump_out_ctr records claimed of dump_out_cap); pairs that must restart go to
// restart (count restart_n).
struct WfaTierIo {
    const int32_t *list;
    const int2 *ents;
    int64_t n;
    const int *n_dev;
    const int64_t *seg;
    int *ctr;
    const uint8_t *dumps_in;
    int64_t dump_in_stride;
    int2 *next;
    int *next_n;
    uint8_t *dumps_out;
    int64_t dump_out_stride, dump_out_cap;
    int *dump_out_ctr;
    int2 *restart;
    int *restart_n;
    int32_t *gring;  // G tier: grid regions of gring_block_bytes
    // exact pruning: per pair a cost no lower than the optimum (-1: max_error), so
    // diagonals k with s + e*|k - target| above it are skipped; and the bound
    // pass's band half-width (> 0: only [min(0, target) - w, max(0, target) + w])
    const int32_t *ubound;
    int32_t band_w;
};
cudaError_t launch_wfa_tier(const WfaTierPlan &pl, int tier, int grid, SeqView q, SeqView r,
                            WfaParams p, const WfaTierIo &io, int32_t *out, int64_t *work,
                            int *err_flag, cudaStream_t st);

// WFA history record of one pair (the CIGAR traceback's input), at a 16-byte
// aligned offset of an arena: int32 header[3 * S] (per visited score index:
// first diagonal a, last diagonal b, offset of its cells in 4-byte words from
// the record start), then per score with a <= b: int32 M-after-extend[w] and
// uint8 decision[w] padded to 4 bytes (w = b - a + 1).  Decision bits: 0-1
// source of M before extension (0 none, 1 mismatch, 2 I, 3 D), bit 2 I comes
// from an I extension (else from an open), bit 3 D comes from a D extension.
__host__ __device__ inline int64_t wfa_hist_cell_bytes(int64_t w) { return 4 * w + ((w + 3) & ~3); }
__host__ __device__ inline int64_t wfa_hist_record_bytes(int64_t cell_bytes, int64_t steps)
{
    return (12 * steps + cell_bytes + 15) & ~int64_t(15);
}

// CIGAR pass over pairs pairs[0..n) (cost and history cell bytes from the
// cost pass, history record at arena + arena_off[pair]; the first n_team
// pairs one per 128-thread block, the rest one per warp; counters[0] and
// counters[32] zeroed); run-length CIGAR ops of pair i go to
// runs[run_off[i] ..], their count to run_count[i].  A run is len << 2 | op
// (op 0 '=', 1 'X', 2 'I', 3 'D').
// Resident 128-thread blocks per SM of the CIGAR kernel.
int wfa_cigar_blocks_per_sm();
cudaError_t launch_wfa_cigar(SeqView q, SeqView r, WfaParams p, const int32_t *pairs, int64_t n,
                             int64_t n_team, int *counters, const int32_t *cost,
                             const int64_t *hist_cells, const int64_t *arena_off, uint8_t *arena,
                             int32_t *scratch, int64_t slot_width, int grid, uint32_t *runs,
                             const int64_t *run_off, int32_t *run_count, int *err_flag,
                             cudaStream_t st);

cudaError_t launch_int_peak(int kind, int grid, int block, int iters, uint32_t *sink,
                            cudaStream_t st);

}  // namespace gb2
