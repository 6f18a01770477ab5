"""Drop-in alignment API with the signatures of genomics/cpu/align_cpu.mojo,
computed on the GPU by libgenomics_b200.so.

smith_waterman_banded(query, reference, cfg) -> AlignResult and
wfa_affine_cpu(query, ref_seq, cfg) -> int keep the reference's names,
argument meaning and results (align_cpu.mojo:75-79, :229-233); each call
uploads, launches and synchronises (the plain per-call path).  The batch
forms take two SequenceBatches and align pair i = (queries[i], refs[i]).
"""
from __future__ import annotations

from dataclasses import dataclass, field
import threading

import numpy as np

from .core import SequenceBatch, SequenceView
from .device import GenomicsDevice


@dataclass
class AlignConfig:
    """align_cpu.mojo:18-25.  Penalties are negative."""
    match_score: int
    mismatch: int
    gap_open: int
    gap_extend: int
    band_width: int


@dataclass
class AlignResult:
    """align_cpu.mojo:28-36 (starts are 0 and the CIGAR empty, :302-309)."""
    score: int
    query_start: int
    ref_start: int
    query_end: int
    ref_end: int
    cigar: list = field(default_factory=list)


@dataclass
class WFAConfig:
    """align_cpu.mojo:62-68.  Positive costs."""
    x: int
    o: int
    e: int
    max_error: int


def default_config() -> AlignConfig:
    """align_cpu.mojo:46-53."""
    return AlignConfig(match_score=2, mismatch=-3, gap_open=-5, gap_extend=-2, band_width=32)


def default_wfa_config() -> WFAConfig:
    """align_cpu.mojo:71-72."""
    return WFAConfig(x=4, o=6, e=2, max_error=200)


_dev = None
_dev_lock = threading.Lock()


def default_device() -> GenomicsDevice:
    global _dev
    with _dev_lock:
        if _dev is None:
            _dev = GenomicsDevice(0)
        return _dev


def smith_waterman_banded(query: SequenceView, reference: SequenceView,
                          cfg: AlignConfig) -> AlignResult:
    """Banded local alignment of one pair (align_cpu.mojo:229-309), on the GPU."""
    s, qe, re_ = default_device().sw_pair(query.packed, query.length, reference.packed,
                                          reference.length, cfg)
    return AlignResult(score=s, query_start=0, ref_start=0, query_end=qe, ref_end=re_, cigar=[])


def needleman_wunsch_banded(query: SequenceView, reference: SequenceView,
                            cfg: AlignConfig) -> AlignResult:
    """Banded global alignment of one pair (align_cpu.mojo:312-377, with the band rows
    sized as its indexing intends), on the GPU: score, ends at (qlen-1, rlen-1)."""
    s, qe, re_ = default_device().nw_pair(query.packed, query.length, reference.packed,
                                          reference.length, cfg)
    return AlignResult(score=s, query_start=0, ref_start=0, query_end=qe, ref_end=re_, cigar=[])


def wfa_affine_cigar_cpu(query: SequenceView, ref_seq: SequenceView, cfg: WFAConfig):
    """Gap-affine WFA with CIGAR traceback of one pair (align_cpu.mojo:380-623), on the
    GPU: (score, CIGAR string); (-1, '') past cfg.max_error."""
    return default_device().wfa_cigar_pair(query.packed, query.length, ref_seq.packed,
                                           ref_seq.length, cfg)


def wfa_affine_cpu(query: SequenceView, ref_seq: SequenceView, cfg: WFAConfig) -> int:
    """Gap-affine WFA cost of one pair, or -1 past cfg.max_error
    (align_cpu.mojo:75-226).  The name is the reference's; it runs on the GPU."""
    return default_device().wfa_pair(query.packed, query.length, ref_seq.packed,
                                     ref_seq.length, cfg)


wfa_affine = wfa_affine_cpu


def sw_banded_batch(queries: SequenceBatch, refs: SequenceBatch, cfg: AlignConfig, bands=None,
                    n_pairs=None, batched: bool = True, device: GenomicsDevice | None = None):
    """Batched banded SW: structured array (score, query_end, ref_end)."""
    dev = device or default_device()
    return dev.sw_banded(queries, refs, cfg, bands=bands, n_pairs=n_pairs, batched=batched)


def wfa_affine_batch(queries: SequenceBatch, refs: SequenceBatch, cfg: WFAConfig,
                     n_pairs=None, batched: bool = True,
                     device: GenomicsDevice | None = None) -> np.ndarray:
    """Batched gap-affine WFA costs (int32, -1 past max_error)."""
    dev = device or default_device()
    return dev.wfa_affine(queries, refs, cfg, n_pairs=n_pairs, batched=batched)
