"""Seeded synthetic workloads (csrc/synth.c) as SequenceBatch pairs.

Workload ids: 0 reads 1 Mbp (150 bp vs 200 bp, band 32); 1 the same over a
10 Mbp reference; 2 WFA pairs 100-10,000 bp at 1-10% divergence; 3 mixed SW
100-2,000 bp, bands {16,32,64,128}, N runs; 4 serving pool; 100 the
reference harness's own LCG pairs (benchmarks/harness.mojo:59-66).
Seeds default to 0xB2000000 + workload id.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _build
from .core import SequenceBatch

GENERATOR_VERSION = 1


class _GsBatch(ctypes.Structure):
    _fields_ = [
        ("q_packed", ctypes.c_void_p), ("q_nmask", ctypes.c_void_p),
        ("q_offsets", ctypes.c_void_p), ("q_lengths", ctypes.c_void_p),
        ("q_words", ctypes.c_int64),
        ("r_packed", ctypes.c_void_p), ("r_nmask", ctypes.c_void_p),
        ("r_offsets", ctypes.c_void_p), ("r_lengths", ctypes.c_void_p),
        ("r_words", ctypes.c_int64),
        ("band", ctypes.c_void_p), ("kind", ctypes.c_void_p), ("n", ctypes.c_int64),
    ]


_synth = None


def _lib():
    global _synth
    if _synth is None:
        if not os.path.exists(_build.SYNTH):
            _build.build()
        L = ctypes.CDLL(_build.SYNTH)
        L.gs_generate.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int64,
                                  ctypes.POINTER(_GsBatch)]
        L.gs_generate.restype = ctypes.c_int
        L.gs_free.argtypes = [ctypes.POINTER(_GsBatch)]
        L.gs_free.restype = None
        _synth = L
    return _synth


def _copy(ptr, n, dtype):
    dtype = np.dtype(dtype)
    if n <= 0 or not ptr:
        return np.zeros(0, dtype)
    buf = (ctypes.c_char * (n * dtype.itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype, count=n).copy()


# Generator of every synthetic workload (csrc/synth.c): a SplitMix64-seeded xoshiro256**
# stream per workload; bump the version when its output for a given seed changes.
GENERATOR = "genomics_synth v1 (SplitMix64-seeded xoshiro256**)"


def default_seed(workload: int) -> int:
    return 0xB2000000 + int(workload)


def generate(workload: int, n: int, seed: int | None = None, param: int = 0, pinned: bool = False):
    """Returns (queries, refs, bands int32[n], kinds int32[n]) for a workload."""
    L = _lib()
    g = _GsBatch()
    s = default_seed(workload) if seed is None else int(seed)
    rc = L.gs_generate(int(workload), int(n), s & 0xFFFFFFFFFFFFFFFF, int(param), ctypes.byref(g))
    if rc != 0:
        raise ValueError(f"unknown workload {workload}")
    try:
        qb = SequenceBatch.from_arrays(_copy(g.q_packed, g.q_words, np.uint64),
                                       _copy(g.q_nmask, g.q_words, np.uint64),
                                       _copy(g.q_offsets, g.n, np.int64),
                                       _copy(g.q_lengths, g.n, np.int64), pinned=pinned)
        rb = SequenceBatch.from_arrays(_copy(g.r_packed, g.r_words, np.uint64),
                                       _copy(g.r_nmask, g.r_words, np.uint64),
                                       _copy(g.r_offsets, g.n, np.int64),
                                       _copy(g.r_lengths, g.n, np.int64), pinned=pinned)
        bands = _copy(g.band, g.n, np.int32)
        kinds = _copy(g.kind, g.n, np.int32)
    finally:
        L.gs_free(ctypes.byref(g))
    return qb, rb, bands, kinds


def sw_cells(queries: SequenceBatch, bands) -> int:
    """SW work in the reference's convention: sum of qlen * (2*band + 1)
    (benchmarks/bench_alignment.mojo:51)."""
    ql = queries.arrays()[3]
    b = np.asarray(bands, np.int64)
    if b.ndim == 0:
        b = np.full(ql.size, int(b), np.int64)
    return int((ql[:b.size] * (2 * b + 1)).sum())


def wfa_max_error_cover(queries: SequenceBatch, refs: SequenceBatch, x: int, o: int, e: int) -> int:
    """Largest per-pair cost bound x*min(q,r) + (q != r) * (o + e*|q-r|) over
    the batch: with it no pair returns -1, and since a larger max_error never
    changes a cost that fits, one batch-wide value gives every pair's cost."""
    ql = queries.arrays()[3]
    rl = refs.arrays()[3]
    n = min(ql.size, rl.size)
    ql, rl = ql[:n], rl[:n]
    bound = x * np.minimum(ql, rl) + np.where(ql != rl, o + e * np.abs(ql - rl), 0)
    return int(bound.max()) if n else 0
