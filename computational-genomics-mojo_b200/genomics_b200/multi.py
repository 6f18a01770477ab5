"""One caller's pair list over several devices.

Pairs are independent (the reference gives each its own thread block,
genomics/gpu/align_gpu.mojo:80), so the list splits into contiguous slices
by cumulative work (gb2_partition_pairs) and nothing crosses between devices
except the results.  Two forms:

* one process, several contexts: sw_banded_multi / wfa_affine_multi run a
  slice per GenomicsDevice (gb2_*_multi) and return results in input order;
* one process per GPU (torchrun): every rank computes the same partition,
  aligns its own slice on its own device (align_slice) and the slices are
  gathered with a torch.distributed all_gather (gather_slices) -- NCCL over
  NVLink for device tensors, gloo on the host.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import SwResult, check
from .core import SequenceBatch
from .device import SW_RESULT_DTYPE, GenomicsDevice, _sw_cfg, _wfa_cfg

SW, WFA = 0, 1


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def partition(q_lengths, r_lengths, n_parts: int, kind: int = SW, band: int = 0,
              bands=None) -> np.ndarray:
    """bounds[0..n_parts]: part k is pairs [bounds[k], bounds[k+1]), cut by cumulative
    work (SW cells qlen*(2*band+1); WFA max(qlen, rlen)^2), as gb2_partition_pairs."""
    ql = np.ascontiguousarray(q_lengths, np.int64)
    rl = np.ascontiguousarray(r_lengths, np.int64)
    n = min(ql.size, rl.size)
    b = None if bands is None else np.ascontiguousarray(bands, np.int32)
    out = np.zeros(n_parts + 1, np.int64)
    check(_lib.lib().gb2_partition_pairs(_p(ql), _p(rl), _p(b), int(band), int(kind), n,
                                         int(n_parts), _p(out)))
    return out


def _ctx_array(devices):
    arr = (ctypes.c_void_p * len(devices))()
    for k, d in enumerate(devices):
        arr[k] = d.ctx
    return arr


def _host_arrays(q: SequenceBatch, r: SequenceBatch):
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    if qp.size == 0:
        qp = np.zeros(1, np.uint64)
    if rp.size == 0:
        rp = np.zeros(1, np.uint64)
    return qp, qo, ql, rp, ro, rl


def sw_banded_multi(devices, q: SequenceBatch, r: SequenceBatch, cfg, bands=None,
                    flags: int = _lib.FLAG_BATCHED) -> np.ndarray:
    """Banded Smith-Waterman over pairs (q[i], r[i]), slice k on devices[k]."""
    qp, qo, ql, rp, ro, rl = _host_arrays(q, r)
    n = min(ql.size, rl.size)
    out = np.zeros(n, SW_RESULT_DTYPE)
    b = None if bands is None else np.ascontiguousarray(bands, np.int32)
    c = _sw_cfg(cfg)
    check(_lib.lib().gb2_sw_banded_multi(_ctx_array(devices), len(devices), _p(qp), _p(qo),
                                         _p(ql), _p(rp), _p(ro), _p(rl), ctypes.byref(c), _p(b),
                                         n, _p(out), int(flags)))
    return out


def wfa_affine_multi(devices, q: SequenceBatch, r: SequenceBatch, cfg,
                     flags: int = _lib.FLAG_BATCHED) -> np.ndarray:
    """Gap-affine WFA costs over pairs (q[i], r[i]), slice k on devices[k]."""
    qp, qo, ql, rp, ro, rl = _host_arrays(q, r)
    n = min(ql.size, rl.size)
    out = np.zeros(n, np.int32)
    c = _wfa_cfg(cfg)
    check(_lib.lib().gb2_wfa_affine_multi(_ctx_array(devices), len(devices), _p(qp), _p(qo),
                                          _p(ql), _p(rp), _p(ro), _p(rl), ctypes.byref(c), n,
                                          _p(out), int(flags)))
    return out


def slice_batch(b: SequenceBatch, i0: int, i1: int) -> SequenceBatch:
    """Sequences [i0, i1) of a batch, sharing its packed words."""
    p, m, o, l = b.arrays()
    return SequenceBatch.from_arrays(p, m, o[i0:i1], l[i0:i1])


def align_slice(dev: GenomicsDevice, q: SequenceBatch, r: SequenceBatch, bounds, rank: int,
                kind: int, cfg, bands=None) -> np.ndarray:
    """This rank's slice on its own device: int32 rows (score, query_end, ref_end) for
    Smith-Waterman, (cost,) for WFA."""
    i0, i1 = int(bounds[rank]), int(bounds[rank + 1])
    qs, rs = slice_batch(q, i0, i1), slice_batch(r, i0, i1)
    if kind == SW:
        res = dev.sw_banded(qs, rs, cfg, bands=None if bands is None else bands[i0:i1])
        return np.ascontiguousarray(res).view(np.int32).reshape(-1, 3)
    return np.asarray(dev.wfa_affine(qs, rs, cfg), np.int32).reshape(-1, 1)


def gather_slices(local: np.ndarray, bounds, group=None, device=None) -> np.ndarray:
    """All ranks' slices of an int32 [rows, width] result, concatenated in rank order
    (= input order) on every rank.  Slices are padded to the longest for all_gather;
    `device` (e.g. "cuda:0") keeps the exchange on the GPU (NCCL)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    sizes = np.diff(np.asarray(bounds, np.int64))
    assert sizes.size == world and local.shape[0] == sizes[dist.get_rank(group)]
    width = local.shape[1]
    cap = int(sizes.max()) if sizes.size else 0
    pad = np.zeros((cap, width), np.int32)
    pad[:local.shape[0]] = local
    t = torch.from_numpy(pad)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return np.concatenate([parts[k].cpu().numpy()[:sizes[k]] for k in range(world)], axis=0)


def align_distributed(dev: GenomicsDevice, q: SequenceBatch, r: SequenceBatch, kind: int, cfg,
                      bands=None, group=None, device=None) -> np.ndarray:
    """One process per GPU: partition by work, align this rank's slice, gather all."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    band = cfg.band_width if kind == SW else 0
    bounds = partition(q.arrays()[3], r.arrays()[3], world, kind, band, bands)
    local = align_slice(dev, q, r, bounds, rank, kind, cfg, bands)
    full = gather_slices(local, bounds, group, device)
    if kind == SW:
        return np.ascontiguousarray(full).view(SW_RESULT_DTYPE).reshape(-1)
    return full[:, 0].copy()


__all__ = ["partition", "sw_banded_multi", "wfa_affine_multi", "slice_batch", "align_slice",
           "gather_slices", "align_distributed", "SW", "WFA"]
