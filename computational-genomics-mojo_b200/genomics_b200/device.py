"""GenomicsDevice: the device context, mirroring genomics/gpu/device.mojo.

The reference's GenomicsDevice (device.mojo:21-138) wraps MAX's
DeviceContext and fills host buffers element by element before each copy.
Here the context lives in libgenomics_b200.so: batches are uploaded once
through pinned staging and stay resident until freed, and the alignment
launchers (launch_banded_sw / launch_wfa_affine, align_gpu.mojo:460-535)
take those resident batches.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FLAG_BATCHED, FLAG_GENERIC, FLAG_INT32, FLAG_PLAIN, SwCfg, WfaCfg, check
from .core import SequenceBatch

SW_RESULT_DTYPE = np.dtype([("score", np.int32), ("query_end", np.int32), ("ref_end", np.int32)])


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


_CIGAR_OPS = "=XID"


def cigar_string(runs) -> str:
    """The reference's CIGAR string from runs (len << 2 | op)."""
    return "".join(f"{int(v) >> 2}{_CIGAR_OPS[int(v) & 3]}" for v in runs)


class DeviceBatch:
    """A SequenceBatch resident in device memory (freed with close())."""

    def __init__(self, dev: "GenomicsDevice", handle, count: int, n_words: int):
        self.dev = dev
        self.handle = handle
        self.count = count
        self.n_words = n_words

    def close(self):
        if self.handle:
            self.dev.L.gb2_batch_free(self.dev.ctx, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _sw_cfg(cfg) -> SwCfg:
    return SwCfg(int(cfg.match_score), int(cfg.mismatch), int(cfg.gap_open),
                 int(cfg.gap_extend), int(cfg.band_width))


def _wfa_cfg(cfg) -> WfaCfg:
    return WfaCfg(int(cfg.x), int(cfg.o), int(cfg.e), int(cfg.max_error))


class GenomicsDevice:
    """One libgenomics_b200 context on one GPU."""

    def __init__(self, device: int = 0):
        self.L = _lib.lib()
        ctx = ctypes.c_void_p()
        check(self.L.gb2_create(int(device), ctypes.byref(ctx)))
        self.ctx = ctx
        self.device = device

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if self.ctx:
            self.L.gb2_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(self.L.gb2_sync(self.ctx), self.ctx)

    def _check(self, rc):
        check(rc, self.ctx)

    # -- uploads (device.mojo:60-108) ----------------------------------------------
    def upload_batch(self, batch: SequenceBatch, with_nmask: bool = True) -> DeviceBatch:
        packed, nm, off, ln = batch.arrays()
        h = ctypes.c_void_p()
        self._check(self.L.gb2_batch_upload(self.ctx, _ptr(packed), packed.size,
                                            _ptr(nm) if with_nmask else None, _ptr(off),
                                            _ptr(ln), ln.size, ctypes.byref(h)))
        return DeviceBatch(self, h, int(ln.size), int(packed.size))

    def batch_from_ascii(self, seqs) -> DeviceBatch:
        """Packs ASCII sequences on the device (SequenceBatch.add_sequence,
        genomics/core/sequence.mojo:38-66); returns the resident batch."""
        bs = [s.encode() if isinstance(s, str) else bytes(s) for s in seqs]
        lengths = np.fromiter((len(b) for b in bs), np.int64, len(bs))
        starts = np.zeros(len(bs), np.int64)
        if len(bs) > 1:
            np.cumsum(lengths[:-1], out=starts[1:])
        buf = np.frombuffer(b"".join(bs) or b"\0", np.uint8)
        h = ctypes.c_void_p()
        self._check(self.L.gb2_batch_from_ascii(self.ctx, _ptr(buf), int(lengths.sum()),
                                                _ptr(starts), _ptr(lengths), len(bs),
                                                ctypes.byref(h)))
        count, words = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.L.gb2_batch_info(h, ctypes.byref(count), ctypes.byref(words)))
        return DeviceBatch(self, h, count.value, words.value)

    def download_batch(self, b: DeviceBatch) -> SequenceBatch:
        """Copies a resident batch back into a host SequenceBatch."""
        p = np.zeros(max(b.n_words, 1), np.uint64)
        m = np.zeros(max(b.n_words, 1), np.uint64)
        o = np.zeros(max(b.count, 1), np.int64)
        ln = np.zeros(max(b.count, 1), np.int64)
        self._check(self.L.gb2_batch_download(self.ctx, b.handle, _ptr(p), _ptr(m), _ptr(o),
                                              _ptr(ln)))
        return SequenceBatch.from_arrays(p[:b.n_words], m[:b.n_words], o[:b.count], ln[:b.count])

    # -- Smith-Waterman -------------------------------------------------------------
    def sw_banded(self, q, r, cfg, bands=None, n_pairs=None, batched=True, flags=0, out=None):
        """Batched smith_waterman_banded over pairs (q[i], r[i]).

        q, r: DeviceBatch (resident) or SequenceBatch (end to end from host
        arrays).  Returns a structured array (score, query_end, ref_end);
        `out` may supply it (e.g. in pinned memory)."""
        n = min(q.count, r.count) if n_pairs is None else int(n_pairs)
        if out is None:
            out = np.zeros(n, SW_RESULT_DTYPE)
        elif out.dtype != SW_RESULT_DTYPE or out.size < n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous SW_RESULT_DTYPE array of n_pairs")
        c = _sw_cfg(cfg)
        fl = flags | (FLAG_BATCHED if batched else FLAG_PLAIN)
        b = None
        if bands is not None:
            b = np.ascontiguousarray(bands, np.int32)
            if b.size < n:
                raise ValueError("bands shorter than n_pairs")
        if isinstance(q, DeviceBatch):
            self._check(self.L.gb2_sw_banded(self.ctx, q.handle, r.handle, ctypes.byref(c),
                                             _ptr(b) if b is not None else None, n, _ptr(out),
                                             fl))
        else:
            qp, _, qo, ql = q.arrays()
            rp, _, ro, rl = r.arrays()
            if n > ql.size or n > rl.size:
                raise ValueError("n_pairs exceeds a batch's sequence count")
            self._check(self.L.gb2_sw_banded_host(self.ctx, _ptr(qp), _ptr(qo), _ptr(ql),
                                                  _ptr(rp), _ptr(ro), _ptr(rl), ctypes.byref(c),
                                                  _ptr(b) if b is not None else None, n,
                                                  _ptr(out), fl))
        return out

    def sw_pair(self, qwords, qlen, rwords, rlen, cfg):
        c = _sw_cfg(cfg)
        res = _lib.SwResult()
        qw = np.ascontiguousarray(qwords, np.uint64)
        rw = np.ascontiguousarray(rwords, np.uint64)
        self._check(self.L.gb2_sw_pair(self.ctx, _ptr(qw), int(qlen), _ptr(rw), int(rlen),
                                       ctypes.byref(c), ctypes.byref(res)))
        return res.score, res.query_end, res.ref_end

    # -- NW -----------------------------------------------------------------------------
    def nw_banded(self, q, r, cfg, bands=None, n_pairs=None, flags=0):
        """Batched needleman_wunsch_banded (align_cpu.mojo:312-377, intended semantics):
        structured array (score, query_end = qlen-1, ref_end = rlen-1)."""
        owned = []
        if not isinstance(q, DeviceBatch):
            q = self.upload_batch(q, with_nmask=False)
            owned.append(q)
        if not isinstance(r, DeviceBatch):
            r = self.upload_batch(r, with_nmask=False)
            owned.append(r)
        try:
            n = min(q.count, r.count) if n_pairs is None else int(n_pairs)
            out = np.zeros(max(n, 1), SW_RESULT_DTYPE)
            b = None if bands is None else np.ascontiguousarray(bands, np.int32)
            self._check(self.L.gb2_nw_banded(self.ctx, q.handle, r.handle,
                                             ctypes.byref(_sw_cfg(cfg)),
                                             _ptr(b) if b is not None else None, n, _ptr(out),
                                             flags))
        finally:
            for bb in owned:
                bb.close()
        return out[:n]

    def nw_pair(self, qwords, qlen, rwords, rlen, cfg):
        res = _lib.SwResult()
        qw = np.ascontiguousarray(qwords, np.uint64)
        rw = np.ascontiguousarray(rwords, np.uint64)
        self._check(self.L.gb2_nw_pair(self.ctx, _ptr(qw), int(qlen), _ptr(rw), int(rlen),
                                       ctypes.byref(_sw_cfg(cfg)), ctypes.byref(res)))
        return res.score, res.query_end, res.ref_end

    # -- WFA ----------------------------------------------------------------------------
    def wfa_affine(self, q, r, cfg, n_pairs=None, batched=True, flags=0, out=None):
        """Batched wfa_affine_cpu over pairs (q[i], r[i]); int32 costs (-1 past
        max_error)."""
        n = min(q.count, r.count) if n_pairs is None else int(n_pairs)
        if out is None:
            out = np.zeros(n, np.int32)
        elif out.dtype != np.int32 or out.size < n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous int32 array of n_pairs")
        c = _wfa_cfg(cfg)
        fl = flags | (FLAG_BATCHED if batched else FLAG_PLAIN)
        if isinstance(q, DeviceBatch):
            self._check(self.L.gb2_wfa_affine(self.ctx, q.handle, r.handle, ctypes.byref(c), n,
                                              _ptr(out), fl))
        else:
            qp, _, qo, ql = q.arrays()
            rp, _, ro, rl = r.arrays()
            if n > ql.size or n > rl.size:
                raise ValueError("n_pairs exceeds a batch's sequence count")
            self._check(self.L.gb2_wfa_affine_host(self.ctx, _ptr(qp), _ptr(qo), _ptr(ql),
                                                   _ptr(rp), _ptr(ro), _ptr(rl),
                                                   ctypes.byref(c), n, _ptr(out), fl))
        return out

    def wfa_cigar(self, q, r, cfg, n_pairs=None, flags=0, raw=False):
        """Batched wfa_affine_cigar_cpu: (costs int32[n], CIGAR strings) for pairs
        (q[i], r[i]); '' where the cost is -1 (align_cpu.mojo:380-623).  raw=True
        returns (costs, runs, run_offsets) instead of strings (run = len << 2 | op)."""
        owned = []
        if not isinstance(q, DeviceBatch):
            q = self.upload_batch(q, with_nmask=False)
            owned.append(q)
        if not isinstance(r, DeviceBatch):
            r = self.upload_batch(r, with_nmask=False)
            owned.append(r)
        try:
            n = min(q.count, r.count) if n_pairs is None else int(n_pairs)
            cost = np.zeros(max(n, 1), np.int32)
            offs = np.zeros(n + 1, np.int64)
            cap = n + 1
            for b in (q, r):
                lens = np.zeros(max(b.count, 1), np.int64)
                self._check(self.L.gb2_batch_download(self.ctx, b.handle, None, None, None,
                                                      _ptr(lens)))
                cap += int(lens[:n].sum())
            runs = np.zeros(cap, np.uint32)
            self._check(self.L.gb2_wfa_cigar(self.ctx, q.handle, r.handle,
                                             ctypes.byref(_wfa_cfg(cfg)), n, _ptr(cost),
                                             _ptr(runs), cap, _ptr(offs), flags))
        finally:
            for b in owned:
                b.close()
        if raw:
            return cost[:n], runs[:offs[n]], offs
        return cost[:n], [cigar_string(runs[offs[i]:offs[i + 1]]) for i in range(n)]

    def wfa_cigar_pair(self, qwords, qlen, rwords, rlen, cfg):
        """Per-pair drop-in for wfa_affine_cigar_cpu: (cost, CIGAR string)."""
        qw = np.ascontiguousarray(qwords, np.uint64)
        rw = np.ascontiguousarray(rwords, np.uint64)
        cap = int(qlen) + int(rlen) + 1
        buf = ctypes.create_string_buffer(8 * cap + 16)
        cost = ctypes.c_int32()
        self._check(self.L.gb2_wfa_cigar_pair(self.ctx, _ptr(qw), int(qlen), _ptr(rw), int(rlen),
                                              ctypes.byref(_wfa_cfg(cfg)), ctypes.byref(cost),
                                              buf, len(buf)))
        return int(cost.value), buf.value.decode()

    def wfa_pair(self, qwords, qlen, rwords, rlen, cfg) -> int:
        c = _wfa_cfg(cfg)
        res = ctypes.c_int32()
        qw = np.ascontiguousarray(qwords, np.uint64)
        rw = np.ascontiguousarray(rwords, np.uint64)
        self._check(self.L.gb2_wfa_pair(self.ctx, _ptr(qw), int(qlen), _ptr(rw), int(rlen),
                                        ctypes.byref(c), ctypes.byref(res)))
        return int(res.value)

    # -- measurement ----------------------------------------------------------------------
    def timer_start(self):
        self._check(self.L.gb2_timer_start(self.ctx))

    def timer_stop(self) -> float:
        ms = ctypes.c_float()
        self._check(self.L.gb2_timer_stop(self.ctx, ctypes.byref(ms)))
        return float(ms.value)

    def stats(self):
        ms = ctypes.c_double()
        launches = ctypes.c_int64()
        work = ctypes.c_int64()
        self._check(self.L.gb2_stats(self.ctx, ctypes.byref(ms), ctypes.byref(launches),
                                     ctypes.byref(work)))
        return {"kernel_ms": ms.value, "launches": launches.value, "work_units": work.value}

    def stats_reset(self):
        self._check(self.L.gb2_stats_reset(self.ctx))

    # -- autotuner ----------------------------------------------------------------------
    def autotune(self, kind, q, r, cfg, n_pairs=None, reps=5, bands=None):
        """gb2_autotune: times every variant of one batched kernel on the resident
        batches (kind "sw": the register kernel of cfg.band_width's class, inside the
        whole mixed call when per-pair `bands` are given; "wfa": the WFA kernel),
        checks they agree, installs the fastest in this context and returns
        {"band_class", "chosen", "candidates": [(variant, median ms), ...]}."""
        k = {"sw": _lib.GB2_TUNE_SW, "wfa": _lib.GB2_TUNE_WFA}[kind]
        c = _sw_cfg(cfg) if k == _lib.GB2_TUNE_SW else _wfa_cfg(cfg)
        n = min(q.count, r.count) if n_pairs is None else int(n_pairs)
        b = None
        if bands is not None:
            b = np.ascontiguousarray(bands, np.int32)
            if b.size < n:
                raise ValueError("bands shorter than n_pairs")
        res = _lib.TuneResult()
        self._check(self.L.gb2_autotune(self.ctx, k, q.handle, r.handle, ctypes.byref(c),
                                        _ptr(b) if b is not None else None, n, int(reps),
                                        ctypes.byref(res)))
        return {"band_class": res.band_class, "chosen": res.chosen,
                "candidates": [(res.variant[i], float(res.ms[i]))
                               for i in range(res.n_candidates)]}

    def tune_set(self, kind, variant, band_class=0):
        k = {"sw": _lib.GB2_TUNE_SW, "wfa": _lib.GB2_TUNE_WFA}[kind]
        self._check(self.L.gb2_tune_set(self.ctx, k, int(band_class), int(variant)))

    def tune_get(self, kind, band_class=0):
        k = {"sw": _lib.GB2_TUNE_SW, "wfa": _lib.GB2_TUNE_WFA}[kind]
        v = ctypes.c_int()
        self._check(self.L.gb2_tune_get(self.ctx, k, int(band_class), ctypes.byref(v)))
        return v.value

    def set_profiling(self, on: bool):
        self._check(self.L.gb2_set_profiling(self.ctx, 1 if on else 0))

    def flush_l2(self):
        self._check(self.L.gb2_flush_l2(self.ctx))

    def int_peak(self, kind: int) -> float:
        g = ctypes.c_double()
        self._check(self.L.gb2_int_peak(self.ctx, int(kind), ctypes.byref(g)))
        return float(g.value)


def launch_banded_sw(device: GenomicsDevice, queries: DeviceBatch, refs: DeviceBatch, cfg,
                     n_pairs=None, bands=None):
    """Counterpart of launch_banded_sw (genomics/gpu/align_gpu.mojo:460-492):
    pairs (queries[i], refs[i]) of resident batches; returns the results."""
    return device.sw_banded(queries, refs, cfg, bands=bands, n_pairs=n_pairs, batched=True)


def launch_wfa_affine(device: GenomicsDevice, queries: DeviceBatch, refs: DeviceBatch, cfg,
                      n_pairs=None):
    """Counterpart of launch_wfa_affine (genomics/gpu/align_gpu.mojo:496-535)
    with runtime penalties."""
    return device.wfa_affine(queries, refs, cfg, n_pairs=n_pairs, batched=True)


__all__ = ["GenomicsDevice", "DeviceBatch", "launch_banded_sw", "launch_wfa_affine",
           "SW_RESULT_DTYPE", "FLAG_BATCHED", "FLAG_PLAIN", "FLAG_INT32", "FLAG_GENERIC"]
