"""Serving: continuous batching of alignment requests (gb2_server_*).

A request is a batch of pairs, each banded Smith-Waterman or gap-affine WFA.
The server admits requests in arrival order under a device-memory budget and
runs groups of them on several executors at once, so requests that arrive
while others are on the GPU start before those finish.  Each result equals
what the batch entry points return for the same pair.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib
from ._lib import Request, ServerCfg, ServerStats, check
from .core import SequenceBatch
from .device import SW_RESULT_DTYPE, GenomicsDevice, _sw_cfg, _wfa_cfg

SW, WFA = 0, 1


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class PendingRequest:
    """A submitted request: its ticket, the arrays it keeps alive, and results."""

    def __init__(self, server, ticket, keep, sw_out, wfa_out, kinds):
        self.server = server
        self.ticket = ticket
        self._keep = keep
        self.sw_out = sw_out
        self.wfa_out = wfa_out
        self.kinds = kinds
        self.latency_ms = None
        self.status = None

    def done(self) -> bool:
        if self.status is not None:
            return True
        d = ctypes.c_int()
        check(self.server.L.gb2_server_poll(self.server.handle, self.ticket, ctypes.byref(d)))
        return bool(d.value)

    def cancel(self):
        """Takes the request out of the queue if it has not started (gb2_server_cancel);
        its wait then raises GenomicsError(GB2_ECANCELED)."""
        check(self.server.L.gb2_server_cancel(self.server.handle, self.ticket),
              self.server.dev.ctx)

    def wait(self, timeout_ms: int = -1):
        """Blocks until done; returns (sw_results, wfa_costs) and sets latency_ms."""
        if self.status is None:
            lat = ctypes.c_double()
            rc = self.server.L.gb2_server_wait(self.server.handle, self.ticket, int(timeout_ms),
                                               ctypes.byref(lat))
            if rc == _lib.GB2_ETIMEOUT:
                raise TimeoutError(f"request {self.ticket} not done after {timeout_ms} ms")
            self.status = rc
            self.latency_ms = lat.value
            check(rc, self.server.dev.ctx)
        return self.sw_out, self.wfa_out


class AlignmentServer:
    """gb2_server over one GenomicsDevice."""

    def __init__(self, device: GenomicsDevice, hbm_budget_bytes: int = 8 << 30,
                 max_inflight_groups: int = 4, max_group_pairs: int = 65536, flags: int = 0):
        self.dev = device
        self.L = _lib.lib()
        cfg = ServerCfg(int(hbm_budget_bytes), int(max_inflight_groups), int(max_group_pairs),
                        int(flags))
        h = ctypes.c_void_p()
        check(self.L.gb2_server_start(device.ctx, ctypes.byref(cfg), ctypes.byref(h)),
              device.ctx)
        self.handle = h
        self._lock = threading.Lock()

    def submit(self, queries: SequenceBatch, refs: SequenceBatch, sw_cfg, wfa_cfg, kinds=None,
               bands=None, n_pairs=None) -> PendingRequest:
        qp, _, qo, ql = queries.arrays()
        rp, _, ro, rl = refs.arrays()
        n = min(ql.size, rl.size) if n_pairs is None else int(n_pairs)
        k = None if kinds is None else np.ascontiguousarray(kinds, np.int32)
        b = None if bands is None else np.ascontiguousarray(bands, np.int32)
        sw_out = np.zeros(n, SW_RESULT_DTYPE)
        wfa_out = np.zeros(n, np.int32)
        if qp.size == 0:
            qp = np.zeros(1, np.uint64)
        if rp.size == 0:
            rp = np.zeros(1, np.uint64)
        req = Request(n, _p(qp), _p(qo), _p(ql), _p(rp), _p(ro), _p(rl), _p(k), _p(b),
                      _sw_cfg(sw_cfg), _wfa_cfg(wfa_cfg), _p(sw_out), _p(wfa_out))
        t = ctypes.c_uint64()
        check(self.L.gb2_server_submit(self.handle, ctypes.byref(req), ctypes.byref(t)),
              self.dev.ctx)
        keep = (qp, qo, ql, rp, ro, rl, k, b)
        return PendingRequest(self, t.value, keep, sw_out, wfa_out, k)

    def hold(self, on: bool = True):
        """Holds (or resumes) admission: queued requests wait, running groups finish."""
        check(self.L.gb2_server_hold(self.handle, 1 if on else 0), self.dev.ctx)

    def stats(self) -> dict:
        st = ServerStats()
        check(self.L.gb2_server_stats_get(self.handle, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def stop(self):
        if self.handle:
            check(self.L.gb2_server_stop(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()
