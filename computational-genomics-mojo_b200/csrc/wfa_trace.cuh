// wfa_trace.cuh -- traceback of a WFA history record into CIGAR runs.
//
// The record (layout in gb2_internal.cuh) holds, per visited score, the
// M-after-extension values and one decision byte per diagonal: M's source
// before extension (1 mismatch, 2 I, 3 D: the first source equal to it in the
// order the reference's traceback tests them, align_cpu.mojo:509-601), bit 2
// set when I came from an extension rather than an open, bit 3 likewise for D.
// The traceback needs only those: in M state at (s, k) the current row is
// M-after[s, k]; the row before extension is M-after[s-x, k] + 1 (mismatch),
// M-after[s'-o-e, k'-1] + 1 + j at the open (s', k') of the I chain of j
// extensions, or M-after[s'-o-e, k'+1] at the open of the D chain; the
// difference is a run of '='.  Then 'X' and (s-x, k), or one 'I' per I cell
// back to M at (s-o-e, k-1), or one 'D' per D cell back to M at (s-o-e,
// k+1); down to score 0, diagonal 0.  Ops come out back to front, merged into
// runs (len << 2 | op, op 0 '=', 1 'X', 2 'I', 3 'D') and reversed at the end,
// which is the reference's run-length encoding (:603-621).
#pragma once
#include <cstdint>

namespace gb2 {

struct WfaHist {
    const uint8_t *rec;
    const int32_t *hdr;
    __device__ __forceinline__ int32_t mafter(int sp, int32_t k) const
    {
        if (sp < 0)
            return -(1 << 30);
        const int32_t a = hdr[3 * sp], b = hdr[3 * sp + 1];
        if (k < a || k > b)
            return -(1 << 30);
        return reinterpret_cast<const int32_t *>(rec)[hdr[3 * sp + 2] + (k - a)];
    }
    __device__ __forceinline__ uint32_t dec(int sp, int32_t k) const
    {
        if (sp < 0)
            return 0;
        const int32_t a = hdr[3 * sp], b = hdr[3 * sp + 1];
        if (k < a || k > b)
            return 0;
        const int64_t off = hdr[3 * sp + 2];
        return rec[(off + (b - a + 1)) * 4 + (k - a)];
    }
};

// Runs of the optimal alignment of cost c (score index c/g, diagonal
// qlen - rlen) into dst[0 .. cap); returns their count, or -1 when the record
// is inconsistent or the runs do not fit.  Sequential (one thread).
__device__ __forceinline__ int64_t wfa_traceback(const uint8_t *rec, int32_t c, int g, int xs,
                                                 int oes, int es, int32_t qlen, int32_t rlen,
                                                 uint32_t *dst, int64_t cap)
{
    const WfaHist h{rec, reinterpret_cast<const int32_t *>(rec)};
    int64_t nrun = 0;
    uint32_t cur_op = 4, cur_len = 0;
    bool bad = false;
    auto emit = [&](uint32_t op, int32_t cnt) {
        if (cnt <= 0)
            return;
        if (op == cur_op) {
            cur_len += (uint32_t)cnt;
            return;
        }
        if (cur_len) {
            if (nrun >= cap) {
                bad = true;
                return;
            }
            dst[nrun++] = cur_len << 2 | cur_op;
        }
        cur_op = op;
        cur_len = (uint32_t)cnt;
    };
    int sp = c / g, mode = 0;
    int32_t k = qlen - rlen, crow = h.mafter(sp, k);
    for (int64_t guard = 4 * ((int64_t)qlen + rlen) + 16; !bad; --guard) {
        if (guard <= 0 || sp < 0) {
            bad = true;
            break;
        }
        if (mode == 0) {
            const uint32_t src = h.dec(sp, k) & 3u;
            int32_t before;
            if (sp == 0) {
                before = 0;  // M[0, 0] = 0 before extension
            } else if (src == 1) {
                before = h.mafter(sp - xs, k) + 1;
            } else if (src == 2) {
                int ssp = sp, j = 0;
                int32_t kk = k;
                while (ssp >= 0 && (h.dec(ssp, kk) & 4u)) {
                    ssp -= es;
                    kk -= 1;
                    ++j;
                }
                before = h.mafter(ssp - oes, kk - 1) + 1 + j;
            } else if (src == 3) {
                int ssp = sp;
                int32_t kk = k;
                while (ssp >= 0 && (h.dec(ssp, kk) & 8u)) {
                    ssp -= es;
                    kk += 1;
                }
                before = h.mafter(ssp - oes, kk + 1);
            } else {
                bad = true;
                break;
            }
            emit(0, crow - before);
            crow = before;
            if (sp == 0) {
                if (k != 0)
                    bad = true;
                break;
            }
            if (src == 1) {
                emit(1, 1);
                sp -= xs;
                crow = h.mafter(sp, k);
            } else {
                mode = (int)src - 1;  // 1: I, 2: D
            }
        } else if (mode == 1) {
            emit(2, 1);
            if (h.dec(sp, k) & 4u) {
                sp -= es;
                k -= 1;
                crow -= 1;
            } else {
                sp -= oes;
                k -= 1;
                crow = h.mafter(sp, k);
                mode = 0;
            }
        } else {
            emit(3, 1);
            if (h.dec(sp, k) & 8u) {
                sp -= es;
                k += 1;
            } else {
                sp -= oes;
                k += 1;
                crow = h.mafter(sp, k);
                mode = 0;
            }
        }
    }
    if (!bad && cur_len) {
        if (nrun >= cap)
            bad = true;
        else
            dst[nrun++] = cur_len << 2 | cur_op;
    }
    if (bad)
        return -1;
    for (int64_t i = 0, j = nrun - 1; i < j; ++i, --j) {
        const uint32_t t = dst[i];
        dst[i] = dst[j];
        dst[j] = t;
    }
    return nrun;
}

}  // namespace gb2
