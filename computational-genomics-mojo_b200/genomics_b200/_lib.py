"""ctypes binding of libgenomics_b200.so (include/genomics_b200.h).

The product path always goes through this library; there is no CPU
fallback.  When the shared object is missing the import of the binding
raises, naming the build step."""
from __future__ import annotations

import ctypes
import os

from . import _build

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
P = ctypes.POINTER
vp = ctypes.c_void_p

GB2_OK = 0
GB2_EINVAL = -1
GB2_ENOMEM = -2
GB2_ECUDA = -3
GB2_ENODEV = -4
GB2_ERANGE = -5
GB2_ETIMEOUT = -6
GB2_ESTATE = -7
GB2_EKERNEL = -8
GB2_ESCRATCH = -9
GB2_ECANCELED = -10
GB2_ALLOC_DEVICE = 1
GB2_ALLOC_PINNED = 2

FLAG_PLAIN = 0x0
FLAG_BATCHED = 0x1
FLAG_INT32 = 0x2
FLAG_GENERIC = 0x4
FLAG_GRAPH = 0x8  # capture resident calls into a CUDA graph and replay it
FLAG_NAIVE = 0x10  # baseline: one thread block per pair, input order, no planning
FLAG_NO_PRUNE = 0x20  # WFA: no bound pass, every reachable diagonal (same results)
FLAG_PACKED = 0x40  # SW: the wide-key packed kernel for small batches too (same results)


class SwCfg(ctypes.Structure):
    """gb2_sw_cfg: AlignConfig (genomics/cpu/align_cpu.mojo:18-25)."""
    _fields_ = [("match_score", c_i32), ("mismatch", c_i32), ("gap_open", c_i32),
                ("gap_extend", c_i32), ("band_width", c_i32)]


class SwResult(ctypes.Structure):
    _fields_ = [("score", c_i32), ("query_end", c_i32), ("ref_end", c_i32)]


class WfaCfg(ctypes.Structure):
    """gb2_wfa_cfg: WFAConfig (genomics/cpu/align_cpu.mojo:62-68)."""
    _fields_ = [("x", c_i32), ("o", c_i32), ("e", c_i32), ("max_error", c_i32)]


GB2_TUNE_SW = 1
GB2_TUNE_WFA = 2
GB2_TUNE_MAX = 16


class TuneResult(ctypes.Structure):
    """gb2_tune_result: candidates, their median times and the installed choice."""
    _fields_ = [("kind", c_i32), ("band_class", c_i32), ("n_candidates", c_i32),
                ("chosen", c_i32), ("variant", c_i32 * GB2_TUNE_MAX),
                ("ms", ctypes.c_float * GB2_TUNE_MAX)]


class Request(ctypes.Structure):
    """gb2_request: one serving request (a batch of SW / WFA pairs)."""
    _fields_ = [("n_pairs", c_i64),
                ("q_packed", vp), ("q_offsets", vp), ("q_lengths", vp),
                ("r_packed", vp), ("r_offsets", vp), ("r_lengths", vp),
                ("kinds", vp), ("bands", vp),
                ("sw_cfg", SwCfg), ("wfa_cfg", WfaCfg),
                ("sw_out", vp), ("wfa_out", vp)]


class ServerCfg(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", c_i64), ("max_inflight_groups", c_i32),
                ("max_group_pairs", c_i32), ("flags", c_i32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", c_i64), ("completed", c_i64), ("failed", c_i64),
                ("pairs_completed", c_i64), ("groups_launched", c_i64),
                ("inflight_bytes", c_i64), ("peak_inflight_bytes", c_i64),
                ("cancelled", c_i64)]


# (name, restype, argtypes) for every entry point of include/genomics_b200.h
SIGNATURES = [
    ("gb2_version", ctypes.c_int, []),
    ("gb2_strerror", ctypes.c_char_p, [ctypes.c_int]),
    ("gb2_create", ctypes.c_int, [ctypes.c_int, P(vp)]),
    ("gb2_destroy", ctypes.c_int, [vp]),
    ("gb2_sync", ctypes.c_int, [vp]),
    ("gb2_last_error", ctypes.c_char_p, [vp]),
    ("gb2_batch_upload", ctypes.c_int, [vp, vp, c_i64, vp, vp, vp, c_i64, P(vp)]),
    ("gb2_batch_free", ctypes.c_int, [vp, vp]),
    ("gb2_batch_info", ctypes.c_int, [vp, P(c_i64), P(c_i64)]),
    ("gb2_batch_from_ascii", ctypes.c_int, [vp, vp, c_i64, vp, vp, c_i64, P(vp)]),
    ("gb2_batch_download", ctypes.c_int, [vp, vp, vp, vp, vp, vp]),
    ("gb2_sw_banded", ctypes.c_int, [vp, vp, vp, P(SwCfg), vp, c_i64, vp, ctypes.c_int]),
    ("gb2_sw_banded_host", ctypes.c_int,
     [vp, vp, vp, vp, vp, vp, vp, P(SwCfg), vp, c_i64, vp, ctypes.c_int]),
    ("gb2_sw_pair", ctypes.c_int, [vp, vp, c_i64, vp, c_i64, P(SwCfg), P(SwResult)]),
    ("gb2_wfa_affine", ctypes.c_int, [vp, vp, vp, P(WfaCfg), c_i64, vp, ctypes.c_int]),
    ("gb2_wfa_affine_host", ctypes.c_int,
     [vp, vp, vp, vp, vp, vp, vp, P(WfaCfg), c_i64, vp, ctypes.c_int]),
    ("gb2_wfa_pair", ctypes.c_int, [vp, vp, c_i64, vp, c_i64, P(WfaCfg), P(c_i32)]),
    ("gb2_nw_banded", ctypes.c_int, [vp, vp, vp, P(SwCfg), vp, c_i64, vp, ctypes.c_int]),
    ("gb2_nw_pair", ctypes.c_int, [vp, vp, c_i64, vp, c_i64, P(SwCfg), P(SwResult)]),
    ("gb2_wfa_cigar", ctypes.c_int,
     [vp, vp, vp, P(WfaCfg), c_i64, vp, vp, c_i64, vp, ctypes.c_int]),
    ("gb2_wfa_cigar_pair", ctypes.c_int,
     [vp, vp, c_i64, vp, c_i64, P(WfaCfg), P(c_i32), ctypes.c_char_p, c_i64]),
    ("gb2_wfa_affine_noalloc", ctypes.c_int,
     [vp, c_i64, vp, vp, vp, c_i64, vp, vp, c_i64, c_i64, P(WfaCfg), c_i64, vp, vp]),
    ("gb2_partition_pairs", ctypes.c_int,
     [vp, vp, vp, c_i32, ctypes.c_int, c_i64, ctypes.c_int, vp]),
    ("gb2_sw_banded_multi", ctypes.c_int,
     [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, P(SwCfg), vp, c_i64, vp, ctypes.c_int]),
    ("gb2_wfa_affine_multi", ctypes.c_int,
     [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, P(WfaCfg), c_i64, vp, ctypes.c_int]),
    ("gb2_server_start", ctypes.c_int, [vp, P(ServerCfg), P(vp)]),
    ("gb2_server_submit", ctypes.c_int, [vp, P(Request), P(ctypes.c_uint64)]),
    ("gb2_server_poll", ctypes.c_int, [vp, ctypes.c_uint64, P(ctypes.c_int)]),
    ("gb2_server_wait", ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int, P(ctypes.c_double)]),
    ("gb2_server_stats_get", ctypes.c_int, [vp, P(ServerStats)]),
    ("gb2_server_stop", ctypes.c_int, [vp]),
    ("gb2_server_hold", ctypes.c_int, [vp, ctypes.c_int]),
    ("gb2_server_cancel", ctypes.c_int, [vp, ctypes.c_uint64]),
    ("gb2_debug_fail_alloc", ctypes.c_int, [ctypes.c_int, c_i64]),
    ("gb2_host_alloc", ctypes.c_int, [c_i64, P(vp)]),
    ("gb2_host_free", ctypes.c_int, [vp]),
    ("gb2_timer_start", ctypes.c_int, [vp]),
    ("gb2_timer_stop", ctypes.c_int, [vp, P(ctypes.c_float)]),
    ("gb2_stats", ctypes.c_int, [vp, P(ctypes.c_double), P(c_i64), P(c_i64)]),
    ("gb2_stats_reset", ctypes.c_int, [vp]),
    ("gb2_autotune", ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, vp, c_i64, ctypes.c_int,
                                    P(TuneResult)]),
    ("gb2_tune_set", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("gb2_tune_get", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, P(ctypes.c_int)]),
    ("gb2_set_profiling", ctypes.c_int, [vp, ctypes.c_int]),
    ("gb2_flush_l2", ctypes.c_int, [vp]),
    ("gb2_int_peak", ctypes.c_int, [vp, ctypes.c_int, P(ctypes.c_double)]),
]

_lib = None


class GenomicsError(RuntimeError):
    """A non-zero status from libgenomics_b200."""

    def __init__(self, code: int, detail: str = ""):
        self.code = code
        name = lib().gb2_strerror(code).decode() if _lib is not None else str(code)
        super().__init__(f"{name} ({code})" + (f": {detail}" if detail else ""))


def lib_path() -> str:
    return _build.LIB


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is missing: build it with __graft_entry__.build() or "
                "python computational-genomics-mojo_b200/genomics_b200/_build.py")
        L = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, ctx=None):
    if rc != GB2_OK:
        detail = ""
        if ctx is not None:
            msg = lib().gb2_last_error(ctx)
            detail = msg.decode() if msg else ""
        raise GenomicsError(rc, detail)
