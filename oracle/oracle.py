"""TEST INFRASTRUCTURE ONLY: ctypes front end of the C oracle (align_oracle.c).

The oracle restates the reference's CPU alignment path
(genomics/cpu/align_cpu.mojo) and its 2-bit packing
(genomics/core/sequence.mojo:38-66).  Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline / reference arm may import this module; the
product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_i64p = ctypes.POINTER(ctypes.c_int64)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)


def build(force: bool = False) -> str:
    """Compile align_oracle.c with the recipe in oracle/Makefile."""
    src = os.path.join(_HERE, "align_oracle.c")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.or_ascii_to_2bit.argtypes = [ctypes.c_int]
        L.or_ascii_to_2bit.restype = ctypes.c_int
        L.or_get_base_export.argtypes = [_u64p, ctypes.c_int64]
        L.or_get_base_export.restype = ctypes.c_int64
        L.or_pack_ascii.argtypes = [ctypes.c_char_p, ctypes.c_int64, _u64p, _u64p]
        L.or_pack_ascii.restype = ctypes.c_int64
        sw_args = [_u64p, ctypes.c_int64, _u64p, ctypes.c_int64] + [ctypes.c_int64] * 5 + [_i64p]
        L.or_sw_banded.argtypes = sw_args
        L.or_sw_banded.restype = None
        L.or_nw_banded.argtypes = sw_args
        L.or_nw_banded.restype = None
        wfa_args = [_u64p, ctypes.c_int64, _u64p, ctypes.c_int64] + [ctypes.c_int64] * 4
        L.or_wfa_affine.argtypes = wfa_args
        L.or_wfa_affine.restype = ctypes.c_int64
        L.or_wfa_affine_envelope.argtypes = wfa_args + [_i64p]
        L.or_wfa_affine_envelope.restype = ctypes.c_int64
        L.or_wfa_cigar.argtypes = wfa_args + [ctypes.c_char_p, ctypes.c_int64]
        L.or_wfa_cigar.restype = ctypes.c_int64
        batch_head = [_u64p, _i64p, _i64p, _u64p, _i64p, _i64p, ctypes.c_int64]
        L.or_sw_batch.argtypes = batch_head + [ctypes.c_int64] * 5 + [_i64p, _i32p, _i32p, _i32p, ctypes.c_int]
        L.or_sw_batch.restype = None
        L.or_nw_batch.argtypes = batch_head + [ctypes.c_int64] * 5 + [_i64p, _i32p, ctypes.c_int]
        L.or_nw_batch.restype = None
        L.or_wfa_batch.argtypes = batch_head + [ctypes.c_int64] * 4 + [ctypes.c_int, _i32p, _i64p, ctypes.c_int]
        L.or_wfa_batch.restype = None
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def pack(seq: str | bytes):
    """add_sequence for one sequence -> (packed u64 words, nmask u64 words)."""
    b = seq.encode() if isinstance(seq, str) else bytes(seq)
    n = (len(b) + 31) // 32
    packed = np.zeros(max(n, 1), np.uint64)
    nmask = np.zeros(max(n, 1), np.uint64)
    lib().or_pack_ascii(b, len(b), _p(packed, _u64p), _p(nmask, _u64p))
    return packed[:n], nmask[:n]


def _words(seq):
    p, _ = pack(seq)
    if p.size == 0:
        p = np.zeros(1, np.uint64)
    return np.ascontiguousarray(p), len(seq)


def sw_banded(q: str, r: str, match=2, mismatch=-3, gap_open=-5, gap_extend=-2, band=32):
    """smith_waterman_banded -> (score, qstart, rstart, qend, rend)."""
    qw, ql = _words(q)
    rw, rl = _words(r)
    out = np.zeros(5, np.int64)
    lib().or_sw_banded(_p(qw, _u64p), ql, _p(rw, _u64p), rl, match, mismatch, gap_open,
                       gap_extend, band, _p(out, _i64p))
    return tuple(int(v) for v in out)


def nw_banded(q: str, r: str, match=2, mismatch=-3, gap_open=-5, gap_extend=-2, band=32):
    qw, ql = _words(q)
    rw, rl = _words(r)
    out = np.zeros(5, np.int64)
    lib().or_nw_banded(_p(qw, _u64p), ql, _p(rw, _u64p), rl, match, mismatch, gap_open,
                       gap_extend, band, _p(out, _i64p))
    return tuple(int(v) for v in out)


def wfa_affine(q: str, r: str, x=4, o=6, e=2, max_error=200, envelope=False):
    qw, ql = _words(q)
    rw, rl = _words(r)
    if envelope:
        work = np.zeros(3, np.int64)
        return int(lib().or_wfa_affine_envelope(_p(qw, _u64p), ql, _p(rw, _u64p), rl, x, o, e,
                                                max_error, _p(work, _i64p)))
    return int(lib().or_wfa_affine(_p(qw, _u64p), ql, _p(rw, _u64p), rl, x, o, e, max_error))


def wfa_cigar(q: str, r: str, x=4, o=6, e=2, max_error=200):
    qw, ql = _words(q)
    rw, rl = _words(r)
    cap = 4 * (ql + rl) + 64
    buf = ctypes.create_string_buffer(cap)
    s = lib().or_wfa_cigar(_p(qw, _u64p), ql, _p(rw, _u64p), rl, x, o, e, max_error, buf, cap)
    return int(s), buf.value.decode()


# ---- batch drivers over SequenceBatch-shaped numpy arrays -----------------

def _batch_ptrs(qp, qoff, qlen, rp, roff, rlen):
    arrs = [np.ascontiguousarray(qp, np.uint64), np.ascontiguousarray(qoff, np.int64),
            np.ascontiguousarray(qlen, np.int64), np.ascontiguousarray(rp, np.uint64),
            np.ascontiguousarray(roff, np.int64), np.ascontiguousarray(rlen, np.int64)]
    if arrs[0].size == 0:
        arrs[0] = np.zeros(1, np.uint64)
    if arrs[3].size == 0:
        arrs[3] = np.zeros(1, np.uint64)
    types = [_u64p, _i64p, _i64p, _u64p, _i64p, _i64p]
    return arrs, [_p(a, t) for a, t in zip(arrs, types)]


def sw_batch(qp, qoff, qlen, rp, roff, rlen, match, mismatch, gap_open, gap_extend, band,
             bands=None, threads=None):
    n = len(qlen)
    keep, ptrs = _batch_ptrs(qp, qoff, qlen, rp, roff, rlen)
    sc = np.zeros(n, np.int32)
    qe = np.zeros(n, np.int32)
    re_ = np.zeros(n, np.int32)
    bp = None
    if bands is not None:
        bands = np.ascontiguousarray(bands, np.int64)
        bp = _p(bands, _i64p)
    lib().or_sw_batch(*ptrs, n, match, mismatch, gap_open, gap_extend, band, bp,
                      _p(sc, _i32p), _p(qe, _i32p), _p(re_, _i32p), threads or os.cpu_count())
    return sc, qe, re_


def nw_batch(qp, qoff, qlen, rp, roff, rlen, match, mismatch, gap_open, gap_extend, band,
             bands=None, threads=None):
    n = len(qlen)
    keep, ptrs = _batch_ptrs(qp, qoff, qlen, rp, roff, rlen)
    sc = np.zeros(n, np.int32)
    bp = None
    if bands is not None:
        bands = np.ascontiguousarray(bands, np.int64)
        bp = _p(bands, _i64p)
    lib().or_nw_batch(*ptrs, n, match, mismatch, gap_open, gap_extend, band, bp,
                      _p(sc, _i32p), threads or os.cpu_count())
    return sc


def wfa_batch(qp, qoff, qlen, rp, roff, rlen, x, o, e, max_error, envelope=True, threads=None):
    """Returns (costs int32[n], work int64[3] = cells, extended bases, scores)."""
    n = len(qlen)
    keep, ptrs = _batch_ptrs(qp, qoff, qlen, rp, roff, rlen)
    out = np.zeros(n, np.int32)
    work = np.zeros(3, np.int64)
    lib().or_wfa_batch(*ptrs, n, x, o, e, max_error, 1 if envelope else 0, _p(out, _i32p),
                       _p(work, _i64p), threads or os.cpu_count())
    return out, work
