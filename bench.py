#!/usr/bin/env python
"""Benchmark of the batched pairwise-alignment path on B200.

Default workload (one "step"): batched banded Smith-Waterman over 1,000,000
seeded synthetic read pairs (150 bp query vs the 200 bp reference window
around its origin, 2% substitutions + 0.5% indels, band 32, scores
+2/-4/-4/-2), one pass of the library over device-resident batches.

  value       GCUPS (cells = sum qlen*(2*band+1), the reference's convention,
              benchmarks/bench_alignment.mojo:51) with inputs resident in HBM;
              CUDA events on the library's own stream around each step, L2
              flushed (256 MB write) between steps.
  e2e         the same metric through the public host API (gb2_sw_banded_host)
              from pinned host arrays: host->device copies of the packed words,
              offsets and lengths and the device->host copy of the results are
              inside the timed region.
  roofline    integer-ALU view of the dominant kernel: cells x ops per cell (11
              int32 ops for the reference recurrence as written; 5.5 when the
              packed int16x2 kernel runs, two cells per lane-op) against the
              lane-op peak measured by the library's own microkernels in the same
              run; DRAM traffic per launch from an ncu capture; an HBM view beside.
  cpu_baseline  the C oracle (restatement of align_cpu.mojo) on a bounded
              sample of the same workload, all host threads.

--impl reference times the reference's CPU algorithm (the oracle port: the
reference is Mojo and cannot be built here) on the same workload and metric.
Multi-GPU (torchrun): each rank aligns its own 1,000,000-pair shard (weak
scaling, no collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "computational-genomics-mojo_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "SW GCUPS & WFA pairs/s, batched vs plain on 1 B200; p50/p99 serve latency"
WORKLOAD = ("batched banded Smith-Waterman, 1,000,000 pairs, 150 bp query vs 200 bp target, "
            "band 32, +2/-4/-4/-2, one persistent launch")
SCORING = (2, -4, -4, -2)
BAND = 32
SW_OPS_PER_CELL = 11  # int32 ops per cell of the reference recurrence (align_cpu.mojo:270-296)
SW_OPS_PER_CELL_PACKED = 5.5  # the same ops on int16x2 lanes: two cells per lane-op
# dram__bytes_read.sum + dram__bytes_write.sum of the dominant kernel per step of this
# workload, from one ncu capture (not measurable inside a timed run): a step runs as 4
# launches of 262,144 pairs; the captured launch read 32.02 MB and wrote 0 B (its 3.1 MB
# of results were still in L2 when it ended), times 4.
SW_PACKED_TRAFFIC_BYTES = 128.1e6
SW_PACKED_TRAFFIC_SOURCE = ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum of one "
                            "262,144-pair launch of sw_pack16_kernel<32>, x 4 launches per step "
                            "(capture of commit 78a5858)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=1_000_000)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-sample", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the oracle check of every result (outside the timed regions)")
    ap.add_argument("--no-peaks", action="store_true", help="skip the integer-throughput probes")
    ap.add_argument("--variant", type=int, default=0, help="kernel variant knob (tuning)")
    ap.add_argument("--plain", action="store_true", help="plain launch instead of the queue")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-band SW, long-pair WFA and per-call measurements")
    ap.add_argument("--wfa-pass", type=int, default=0, metavar="N",
                    help="(profiling) one batched WFA pass over N pairs of the long-pair "
                         "WFA workload, then exit")
    return ap.parse_args()


def wfa_pass(n):
    """One batched WFA pass (x4 o6 e2, exact-cover max_error) over the first n pairs of
    the long-pair workload, timed with CUDA events after one warm-up pass and an L2
    flush: the command the WFA profiles use."""
    from genomics_b200 import GenomicsDevice, WFAConfig, synth
    dev = GenomicsDevice(0)
    q, r, _, _ = synth.generate(2, n)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    cfg = WFAConfig(4, 6, 2, me)
    dq, dr = dev.upload_batch(q, with_nmask=False), dev.upload_batch(r, with_nmask=False)
    dev.wfa_affine(dq, dr, cfg, batched=True)  # warm-up: buffers, module load
    dev.stats_reset()
    dev.flush_l2()
    dev.timer_start()
    out = dev.wfa_affine(dq, dr, cfg, batched=True)
    ms = dev.timer_stop()
    assert (out >= 0).all()
    print(json.dumps({"wfa_pass_pairs": n, "max_error": me, "ms": round(ms, 3),
                      "pairs_per_s": round(n / (ms * 1e-3), 1),
                      "wavefront_cells": dev.stats()["work_units"]}), flush=True)
    dq.close()
    dr.close()
    dev.close()


# ---------------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        self.t0 = time.time()

    def stop(self):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        rows = []
        if self.path and os.path.exists(self.path):
            for row in csv.reader(io.StringIO(open(self.path).read())):
                if len(row) >= 9:
                    rows.append([c.strip() for c in row])
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------------
# CPU side (oracle = restatement of align_cpu.mojo)
# ---------------------------------------------------------------------------------
def cpu_sw_gcups(q, r, n_sample: int, threads: int):
    import oracle as O
    O.build()
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    n = min(n_sample, ql.size)
    t = time.perf_counter()
    O.sw_batch(qp, qo[:n], ql[:n], rp, ro[:n], rl[:n], *SCORING, BAND, threads=threads)
    dt = time.perf_counter() - t
    cells = int((ql[:n] * (2 * BAND + 1)).sum())
    return cells / dt / 1e9, n, dt


def cpu_steps(q, r, sample: int, steps: int, warmup: int, threads: int):
    """The oracle (restatement of align_cpu.mojo) on the first `sample` pairs per step:
    `warmup` untimed steps on up to 5,000 pairs, then `steps` timed steps.  Returns
    (GCUPS over the timed steps, total seconds).  The reference arm and the in-run
    cpu_baseline both use it, so their figures are the same measurement."""
    for _ in range(warmup):
        cpu_sw_gcups(q, r, min(sample, 5000), threads)
    ql = q.arrays()[3]
    per_step_cells = int((ql[:sample] * (2 * BAND + 1)).sum())
    total = 0.0
    for _ in range(steps):
        total += cpu_sw_gcups(q, r, sample, threads)[2]
    return per_step_cells * steps / total / 1e9, total


def sw_parity(q, r, got, scoring, band, threads, bands=None):
    """'equal/total' of every pair's (score, query_end, ref_end) against the oracle."""
    import oracle as O
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    sc, qe, re_ = O.sw_batch(qp, qo, ql, rp, ro, rl, *scoring, band, bands=bands,
                             threads=threads)
    ok = (got["score"] == sc) & (got["query_end"] == qe) & (got["ref_end"] == re_)
    return f"{int(ok.sum())}/{ok.size}"


def wfa_parity(q, r, got, cfg, threads):
    """'equal/total' of every pair's cost against the oracle (live-envelope form)."""
    import oracle as O
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    want, _ = O.wfa_batch(qp, qo, ql, rp, ro, rl, cfg.x, cfg.o, cfg.e, cfg.max_error,
                          envelope=True, threads=threads)
    return f"{int((want == got).sum())}/{want.size}"


def workload_config(args, cells, seed):
    """The `config` object of both arms' lines: the same workload, named by its sizes."""
    from genomics_b200 import synth
    return {"workload": WORKLOAD, "pairs_per_gpu": args.pairs, "band": BAND,
            "query_bp": 150, "target_bp": 200, "scoring": list(SCORING),
            "path": "plain" if args.plain else "batched", "variant": args.variant,
            "l2": "flushed between timed steps (256 MB device write)",
            "cells_per_step_per_gpu": int(cells),
            "generator": synth.GENERATOR, "seed": hex(seed),
            "seed_rule": "0xb2000001 + 7919 * rank"}


def reference_arm(args, dist: Dist):
    """The reference's CPU algorithm, timed on this host's cores."""
    if dist.rank != 0:
        dist.close()
        return
    from genomics_b200 import synth
    threads = os.cpu_count() or 1
    q, r, _, _ = synth.generate(1, args.pairs)
    sample = min(args.pairs, max(1000, args.cpu_sample // 2))
    value, total = cpu_steps(q, r, sample, args.steps, args.warmup, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GCUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": workload_config(args, synth.sw_cells(q, BAND), synth.default_seed(1)),
        "note": "the reference is Mojo-only (no toolchain here); its CPU algorithm runs as "
                "the C restatement in oracle/, each step a bounded sample of the workload",
        "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads,
                         "kind": "port",
                         "sample": f"first {sample} of the {args.pairs} pairs per step"},
        "e2e": {"value": round(value, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------
def our_arm(args, dist: Dist):
    from genomics_b200 import AlignConfig, GenomicsDevice, synth
    from genomics_b200.core import pinned_empty
    from genomics_b200.device import SW_RESULT_DTYPE

    dev = GenomicsDevice(dist.local_rank)
    seed = synth.default_seed(1) + 7919 * dist.rank
    q, r, bands, _ = synth.generate(1, args.pairs, seed=seed, pinned=True)
    cfg = AlignConfig(*SCORING, BAND)
    cells = synth.sw_cells(q, BAND)
    flags = args.variant << 8
    batched = not args.plain

    class _Owner:
        _pinned_blocks = []

    owner = _Owner()
    out = pinned_empty(args.pairs * SW_RESULT_DTYPE.itemsize, np.uint8, owner).view(SW_RESULT_DTYPE)

    dq, dr = dev.upload_batch(q, with_nmask=False), dev.upload_batch(r, with_nmask=False)
    for _ in range(max(args.warmup, 3)):
        dev.flush_l2()
        dev.sw_banded(dq, dr, cfg, batched=batched, flags=flags, out=out)

    clocks = Clocks(dist.local_rank)
    dev.stats_reset()
    dev.set_profiling(True)
    dist.barrier()
    dev.synchronize()
    clocks.start()
    times = []
    for _ in range(args.steps):
        dev.flush_l2()
        dev.timer_start()
        dev.sw_banded(dq, dr, cfg, batched=batched, flags=flags, out=out)
        times.append(dev.timer_stop())
    dev.synchronize()
    clk = clocks.stop()
    dist.barrier()
    st = dev.stats()
    dev.set_profiling(False)
    total_ms = sum(times)
    max_ms = dist.max(total_ms)
    kernel_ms = st["kernel_ms"] / args.steps  # dominant (class) kernels per step
    launches = int(st["launches"])
    value = dist.world * args.steps * cells / (max_ms * 1e-3) / 1e9

    # results sanity (bit-exactness is the tests' job)
    assert (out["score"] <= 2 * 150).all() and (out["score"] >= 0).all()

    # e2e: public host API from pinned host arrays
    # bytes the host pipeline copies: the packed words and, for these contiguous batches,
    # int32 lengths (offsets are rebuilt on the device)
    h2d = q.packed.nbytes + r.packed.nbytes + 4 * (q.lengths.size + r.lengths.size)
    d2h = args.pairs * SW_RESULT_DTYPE.itemsize
    e2e_value = None
    if args.e2e_steps > 0:
        dev.sw_banded(q, r, cfg, batched=batched, flags=flags, out=out)  # warm the pipeline
        dist.barrier()
        e2e_t = []
        for _ in range(args.e2e_steps):
            dev.synchronize()
            t = time.perf_counter()
            dev.sw_banded(q, r, cfg, batched=batched, flags=flags, out=out)
            e2e_t.append(time.perf_counter() - t)
        e2e_total = dist.max(sum(e2e_t))
        e2e_value = dist.world * args.e2e_steps * cells / e2e_total / 1e9

    line = None
    if dist.rank == 0:
        peaks = {}
        if not args.no_peaks:
            for kind, name in ((0, "iadd"), (1, "imnmx"), (2, "viaddmax_s32"),
                               (3, "viaddmax_s16x2"), (4, "vimax3_s32"), (5, "lop3"),
                               (6, "imad"), (7, "shfl")):
                peaks[name] = round(dev.int_peak(kind), 1)
            # int32 lane-op peak: plain ALU ops, DPX add-max counted as two ops
            peak_ops = max(peaks["iadd"], peaks["imnmx"], 2 * peaks["viaddmax_s32"])
        else:
            peak_ops = 36600.0  # 148 SMs x 64 lanes x 2 ops (DPX add-max) x 1.965 GHz
        kern_gcups = cells / (kernel_ms * 1e-3) / 1e9
        # the packed int16x2 kernel takes every pair of this workload (band <= 32,
        # score bound match*150 <= 511)
        packed = BAND <= 32 and SCORING[0] * 150 <= 511
        ops_per_cell = SW_OPS_PER_CELL_PACKED if packed else SW_OPS_PER_CELL
        achieved_ops = kern_gcups * ops_per_cell
        # the kernel reads the packed words and int64 offsets and lengths, writes results
        alg_bytes = q.packed.nbytes + r.packed.nbytes + 32 * args.pairs + d2h
        mp = {}
        mp_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(mp_path):
            mp = json.load(open(mp_path))
        hbm_peak = mp.get("hbm_gbs", 6650.0)
        cpu = None
        parity = None
        if args.gpus == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sample = min(args.pairs, max(1000, args.cpu_sample // 2))
            csteps = 5
            g, dt = cpu_steps(q, r, sample, csteps, 3, threads)
            g1, n1, dt1 = cpu_sw_gcups(q, r, max(1000, args.cpu_sample // 5), 1)
            cpu = {"value": round(g, 4), "unit": "GCUPS", "cores": threads, "kind": "port",
                   "sample": f"first {sample} of the {args.pairs} pairs per step, {csteps} "
                             f"timed steps after 3 warm-up steps ({dt:.1f} s), as the "
                             "reference arm",
                   "single_thread": {"value": round(g1, 4), "unit": "GCUPS", "cores": 1,
                                     "sample": f"first {n1} pairs ({dt1:.1f} s), the "
                                               "reference's serial loop"}}
            if not args.no_parity:
                # the oracle as the checker: every pair of the timed step's results
                parity = {"config1_1M_reads": sw_parity(q, r, out, SCORING, BAND, threads)}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GCUPS",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "int16x2" if packed else "int32", "data": "synthetic",
            "config": workload_config(args, cells, seed),
            "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "GCUPS",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "roofline": {"bound": "int_alu", "achieved": round(achieved_ops, 1),
                         "peak": peak_ops, "unit": "Gop/s",
                         "frac": round(achieved_ops / peak_ops, 4),
                         "ops_per_cell": ops_per_cell,
                         "kernel": "sw_pack16_kernel<32>" if packed else "sw_band_kernel<32>",
                         "kernel_ms": round(kernel_ms, 4),
                         "kernel_ms_is": "device span per step of its launches (a 1M-pair "
                                         "step runs as 4 overlapping parts on 2 streams)",
                         "kernel_gcups": round(kern_gcups, 2),
                         "peak_source": "gb2_int_peak microkernels in this run: "
                                        "max(IADD, IMNMX, 2 x DPX viaddmax) lane-ops/s",
                         "traffic": SW_PACKED_TRAFFIC_BYTES if packed else None,
                         "traffic_unit": "bytes per step, 4 launches (ncu)",
                         "traffic_source": SW_PACKED_TRAFFIC_SOURCE if packed else None,
                         "hbm": {"achieved": round(alg_bytes / (kernel_ms * 1e-3) / 1e9, 2),
                                 "peak": hbm_peak, "unit": "GB/s",
                                 "frac": round(alg_bytes / (kernel_ms * 1e-3) / 1e9 / hbm_peak, 5),
                                 "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}},
            "int_peaks_gops": peaks,
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clk,
        }
    dq.close()
    dr.close()
    if line is not None and dist.world == 1 and not args.no_extras:
        line["extras"] = extras(args, dev, line["roofline"]["peak"],
                                line["roofline"]["hbm"]["peak"])
    dev.close()
    dist.close()
    if line:
        print(json.dumps(line), flush=True)


class _PinnedOwner:
    """Keeps page-locked host blocks alive as long as the arrays that use them."""
    def __init__(self):
        self._pinned_blocks = []


def _time_steps(dev, fn, steps, warmup):
    """Device time (ms) per step of fn() on the library stream, L2 flushed between."""
    for _ in range(warmup):
        dev.flush_l2()
        fn()
    ts = []
    for _ in range(steps):
        dev.flush_l2()
        dev.timer_start()
        fn()
        ts.append(dev.timer_stop())
    return statistics.median(ts)


def extras(args, dev, peak_ops, hbm_peak):
    """Batched queue vs plain launch vs per-call drop-in on the mixed-length workloads,
    with the CPU restatement of the reference beside each (all host threads)."""
    import oracle as O
    from genomics_b200 import AlignConfig, WFAConfig, synth
    from genomics_b200._lib import FLAG_NAIVE, FLAG_NO_PRUNE
    from genomics_b200.core import pinned_empty
    from genomics_b200.device import SW_RESULT_DTYPE
    O.build()
    threads = os.cpu_count() or 1
    out = {}
    # each band class alone: the 1,000,000 reads of the headline workload with one band
    # for every pair (bands 16/32 take the narrow-key packed kernel, 64/128 the wide-key one)
    q1, r1, _, _ = synth.generate(1, 1_000_000)
    d1q, d1r = dev.upload_batch(q1, with_nmask=False), dev.upload_batch(r1, with_nmask=False)
    own1 = _PinnedOwner()
    out1 = pinned_empty(q1.count * SW_RESULT_DTYPE.itemsize, np.uint8, own1).view(SW_RESULT_DTYPE)
    classes = {}
    for band in (16, 32, 64, 128):
        cfg_b = AlignConfig(*SCORING, band)
        tcb = _time_steps(dev, lambda: dev.sw_banded(d1q, d1r, cfg_b, batched=True, out=out1),
                          5, 3)
        cells_b = synth.sw_cells(q1, band)
        classes[f"band_{band}"] = {"gcups": round(cells_b / tcb / 1e6, 1), "ms": round(tcb, 3),
                                   "kernel": f"sw_pack16_kernel<{band}, "
                                             f"{'narrow' if band <= 32 else 'wide'} keys>"}
    out["sw_band_classes_1M_reads"] = {
        "workload": "the 1,000,000 reads of the headline workload (150 vs 200 bp, "
                    "+2/-4/-4/-2), one band for every pair, resident, results into "
                    "page-locked memory",
        **classes}
    d1q.close()
    d1r.close()
    # mixed-band SW: 200,000 pairs, 100-2,000 bp, bands {16,32,64,128}, N runs
    q, r, bands, _ = synth.generate(3, 200_000)
    cfg = AlignConfig(*SCORING, 32)
    cells = synth.sw_cells(q, bands)
    dq, dr = dev.upload_batch(q, with_nmask=False), dev.upload_batch(r, with_nmask=False)
    # the per-pair bands in and the results out through page-locked host arrays, as the
    # headline's results are (a pageable array adds a host copy inside the timed region)
    own = _PinnedOwner()
    pbands = pinned_empty(bands.size, np.int32, own)
    pbands[:] = bands
    sw_out = pinned_empty(bands.size * SW_RESULT_DTYPE.itemsize, np.uint8, own).view(SW_RESULT_DTYPE)
    tb = _time_steps(dev, lambda: dev.sw_banded(dq, dr, cfg, bands=pbands, batched=True,
                                                out=sw_out), 10, 5)
    tp = _time_steps(dev, lambda: dev.sw_banded(dq, dr, cfg, bands=pbands, batched=False,
                                                out=sw_out), 10, 5)
    tn = _time_steps(dev, lambda: dev.sw_banded(dq, dr, cfg, bands=pbands, batched=False,
                                                flags=FLAG_NAIVE, out=sw_out), 2, 1)
    res_b = np.array(dev.sw_banded(dq, dr, cfg, bands=pbands, batched=True, out=sw_out))
    m = 3000
    t0 = time.perf_counter()
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    for i in range(m):
        c_i = AlignConfig(*SCORING, int(bands[i]))
        dev.sw_pair(qp[qo[i]:qo[i] + (ql[i] + 31) // 32], int(ql[i]),
                    rp[ro[i]:ro[i] + (rl[i] + 31) // 32], int(rl[i]), c_i)
    tcall = time.perf_counter() - t0
    call_cells = int((ql[:m] * (2 * bands[:m].astype(np.int64) + 1)).sum())
    ns = 20_000
    t0 = time.perf_counter()
    O.sw_batch(qp, qo[:ns], ql[:ns], rp, ro[:ns], rl[:ns], *SCORING, 32, bands=bands[:ns],
               threads=threads)
    tcpu = time.perf_counter() - t0
    cpu_cells = int((ql[:ns] * (2 * bands[:ns].astype(np.int64) + 1)).sum())
    out["mixed_sw_200k"] = {
        "workload": "200,000 pairs, query 100-2,000 bp, target 1.25x, bands {16,32,64,128}, "
                    "1-8% divergence, 1% N runs, +2/-4/-4/-2",
        "cells": cells,
        "batched_gcups": round(cells / tb / 1e6, 2), "batched_ms": round(tb, 3),
        "plain_launch_gcups": round(cells / tp / 1e6, 2), "plain_launch_ms": round(tp, 3),
        "naive_launch_gcups": round(cells / tn / 1e6, 2), "naive_launch_ms": round(tn, 3),
        "naive_is": "one 128-thread block per pair, input order, no planning (GB2_FLAG_NAIVE)",
        "per_call_gcups": round(call_cells / tcall / 1e9, 3),
        "per_call_pairs_per_s": round(m / tcall, 1),
        "batched_over_per_call": round((cells / tb / 1e6) / (call_cells / tcall / 1e9), 1),
        "cpu_gcups": round(cpu_cells / tcpu / 1e9, 3), "cpu_cores": threads,
        "cpu_sample": f"first {ns} pairs",
    }
    if not args.no_parity:
        out["mixed_sw_200k"]["parity"] = sw_parity(q, r, res_b, SCORING, 32, threads,
                                                   bands=bands)
    # autotuner: the register-kernel shape of each band class, tuned inside the
    # whole mixed batch (one class after another), then the batch timed again
    from genomics_b200 import autotune
    table = autotune.tune(dev, dq, dr, sw_cfg=cfg, reps=3, pair_bands=bands)
    tt = _time_steps(dev, lambda: dev.sw_banded(dq, dr, cfg, bands=pbands, batched=True,
                                                out=sw_out), 10, 5)
    out["mixed_sw_200k"]["autotuned"] = {
        "table": table["sw"], "candidates_ms": table["measurements"],
        "tuned_on": "the whole 200,000-pair mixed call, one band class after another",
        "batched_gcups": round(cells / tt / 1e6, 2), "batched_ms": round(tt, 3)}
    autotune.install(dev, {"sw": {str(b): 0 for b in autotune.SW_BANDS}})
    dq.close()
    dr.close()
    # long WFA: 100,000 pairs, 100-10,000 bp, 1-10% divergence, x4 o6 e2
    q, r, _, _ = synth.generate(2, 100_000)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    wcfg = WFAConfig(4, 6, 2, me)
    dq, dr = dev.upload_batch(q, with_nmask=False), dev.upload_batch(r, with_nmask=False)
    n = 100_000
    wout = pinned_empty(n, np.int32, own)
    dev.stats_reset()
    tb = _time_steps(dev, lambda: dev.wfa_affine(dq, dr, wcfg, batched=True, out=wout), 2, 1)
    wcells = dev.stats()["work_units"] // 3
    wres = np.array(dev.wfa_affine(dq, dr, wcfg, batched=True))
    # the envelope the algorithm defines (every diagonal the sources reach, no bound
    # pruning): the algorithmic work the roofline counts, and that path's time
    dev.stats_reset()
    tnp = _time_steps(dev, lambda: dev.wfa_affine(dq, dr, wcfg, batched=True,
                                                  flags=FLAG_NO_PRUNE, out=wout), 1, 1)
    ecells = dev.stats()["work_units"] // 2
    tp = _time_steps(dev, lambda: dev.wfa_affine(dq, dr, wcfg, batched=False, out=wout), 2, 1)
    tn = _time_steps(dev, lambda: dev.wfa_affine(dq, dr, wcfg, batched=False,
                                                 flags=FLAG_NAIVE, out=wout), 1, 1)
    # the single-kernel design with rings in global memory (tuning variant 5: five
    # 4-warp blocks per SM, length-sorted queue) for comparison
    tg = _time_steps(dev, lambda: dev.wfa_affine(dq, dr, wcfg, batched=True, flags=5 << 8,
                                                 out=wout), 1, 1)
    w200 = WFAConfig(4, 6, 2, 200)
    t200 = _time_steps(dev, lambda: dev.wfa_affine(dq, dr, w200, batched=True, out=wout), 2, 1)
    c200 = dev.wfa_affine(dq, dr, w200, batched=True)
    wbytes = q.packed.nbytes + r.packed.nbytes + 20 * n
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    m = 300
    t0 = time.perf_counter()
    for i in range(m):
        dev.wfa_pair(qp[qo[i]:qo[i] + (ql[i] + 31) // 32], int(ql[i]),
                     rp[ro[i]:ro[i] + (rl[i] + 31) // 32], int(rl[i]), wcfg)
    tcall = time.perf_counter() - t0
    # CPU: a seeded sample stratified by length decile, 16 pairs per decile (lengths
    # are log-uniform, so each decile holds a tenth of the pairs and the sample's rate
    # is the workload's)
    lmax = np.maximum(ql, rl)
    edges = np.quantile(lmax, np.linspace(0, 1, 11))
    srng = np.random.default_rng(0xB2000002)
    idx = np.concatenate([srng.choice(np.nonzero((lmax >= edges[d]) & (lmax <= edges[d + 1]))[0],
                                      16, replace=False) for d in range(10)])
    ns = idx.size
    t0 = time.perf_counter()
    O.wfa_batch(qp, qo[idx], ql[idx], rp, ro[idx], rl[idx], 4, 6, 2, me, envelope=False,
                threads=threads)
    tcpu = time.perf_counter() - t0
    out["wfa_100k"] = {
        "workload": "100,000 pairs, 100-10,000 bp log-uniform, 1-10% divergence (70% subst., "
                    "30% indels), x4 o6 e2",
        "max_error": me, "max_error_rule": "largest per-pair exact-cover bound (no pair -1)",
        "wavefront_cells": int(ecells),
        "executed_cells": int(wcells),
        "executed_cells_are": "cells the tiers computed: the envelope less what the exact "
                              "bound pruning skips, plus the bound pass's own cells",
        "no_prune_ms": round(tnp, 3),
        "batched_pairs_per_s": round(n / (tb * 1e-3), 1), "batched_ms": round(tb, 3),
        "plain_launch_pairs_per_s": round(n / (tp * 1e-3), 1), "plain_launch_ms": round(tp, 3),
        "naive_launch_pairs_per_s": round(n / (tn * 1e-3), 1), "naive_launch_ms": round(tn, 3),
        "naive_is": "one 4-warp block per pair, input order, rings in global memory, no "
                    "planning (GB2_FLAG_NAIVE)",
        "global_ring_kernel_ms": round(tg, 3),
        "per_call_pairs_per_s": round(m / tcall, 1),
        "batched_over_per_call": round((n / (tb * 1e-3)) / (m / tcall), 1),
        "cpu_pairs_per_s": round(ns / tcpu, 2), "cpu_cores": threads,
        "cpu_sample": f"{ns} pairs, 16 per length decile (seeded), statement-for-statement "
                      f"port (per-score reset of 2*max_error+1 diagonals, as the reference)",
        # 13 int ops per wavefront cell: I 3, D 1, M 3, one extend step 6
        "roofline": {"bound": "instruction issue of dependent chains per score step "
                              "(rings in shared memory)",
                     "ops_per_cell": 13,
                     "cells_counted": "the envelope (wavefront_cells)",
                     "achieved": round(ecells * 13 / (tb * 1e-3) / 1e9, 1),
                     "peak": peak_ops, "unit": "Gop/s",
                     "frac": round(ecells * 13 / (tb * 1e-3) / 1e9 / peak_ops, 4),
                     # bytes: both sequences' packed words + 20 B of offsets, lengths
                     # and the cost per pair
                     "hbm": {"bytes": int(wbytes),
                             "achieved": round(wbytes / (tb * 1e-3) / 1e9, 2),
                             "peak": hbm_peak, "unit": "GB/s",
                             "frac": round(wbytes / (tb * 1e-3) / 1e9 / hbm_peak, 6)}},
        "parity": None if args.no_parity else wfa_parity(q, r, wres, wcfg, threads),
        "max_error_200": {"pairs_per_s": round(n / (t200 * 1e-3), 1), "ms": round(t200, 3),
                          "pairs_minus_one": int((c200 < 0).sum()),
                          "note": "the reference's default budget: most long pairs exceed "
                                  "it and return -1"},
    }
    # WFA with CIGAR traceback: the first 20,000 pairs of the same workload
    nc = 20_000
    qc, rc_, _, _ = synth.generate(2, nc)
    mec = synth.wfa_max_error_cover(qc, rc_, 4, 6, 2)
    ccfg = WFAConfig(4, 6, 2, mec)
    dqc, drc = dev.upload_batch(qc, with_nmask=False), dev.upload_batch(rc_, with_nmask=False)
    tcig = _time_steps(dev, lambda: dev.wfa_cigar(dqc, drc, ccfg, raw=True), 2, 1)
    _, runs, _ = dev.wfa_cigar(dqc, drc, ccfg, raw=True)
    # CPU: the oracle's restatement of wfa_affine_cigar_cpu keeps four int64 arrays of
    # (max_error+1) x (2 max_error+1); it runs with max_error = each pair's own cost (the
    # smallest budget that finds it) on the first pairs whose cost is at most 1,500
    qp, _, qo, ql = qc.arrays()
    rp, _, ro, rl = rc_.arrays()
    costs = dev.wfa_affine(dqc, drc, ccfg)
    sample = [i for i in range(nc) if costs[i] <= 1500][:20]
    strs = lambda p_, o_, l_: "".join("ACGT"[(int(p_[o_ + k // 32]) >> (62 - 2 * (k % 32))) & 3]
                                      for k in range(int(l_)))
    pairs = [(strs(qp, qo[i], ql[i]), strs(rp, ro[i], rl[i]), int(costs[i])) for i in sample]
    t0 = time.perf_counter()
    for a, b, c in pairs:
        O.wfa_cigar(a, b, 4, 6, 2, c)
    tcc = time.perf_counter() - t0
    out["wfa_cigar_20k"] = {
        "workload": "first 20,000 pairs of the long-pair WFA workload, x4 o6 e2, exact-cover "
                    "max_error; cost + CIGAR runs back on the host",
        "max_error": mec, "cigar_runs": int(runs.size),
        "gpu_pairs_per_s": round(nc / (tcig * 1e-3), 1), "gpu_ms": round(tcig, 3),
        "cpu_pairs_per_s": round(len(pairs) / tcc, 2), "cpu_cores": 1,
        "cpu_sample": f"{len(pairs)} pairs with cost <= 1500, oracle restatement of "
                      f"wfa_affine_cigar_cpu with max_error = each pair's cost",
    }
    dqc.close()
    drc.close()
    # banded Needleman-Wunsch: the 1,000,000 reads against the 150 bp window of the
    # reference at their origin (the default targets' bases 25-174), band 32, so the
    # global alignment's end cell lies on the band's centre diagonal (with the 200 bp
    # targets it would lie 50 diagonals off, outside the band, and every score would
    # be the reference's -1,000,000)
    qn, rfull, _, _ = synth.generate(1, 1_000_000)
    rn = _window_batch(rfull, 25, 150)
    ncfg = AlignConfig(2, -4, -4, -2, 32)
    ncells = synth.sw_cells(qn, 32)
    dqn, drn = dev.upload_batch(qn, with_nmask=False), dev.upload_batch(rn, with_nmask=False)
    tnw = _time_steps(dev, lambda: dev.nw_banded(dqn, drn, ncfg), 3, 2)
    qp, _, qo, ql = qn.arrays()
    rp, _, ro, rl = rn.arrays()
    ns = 100_000
    t0 = time.perf_counter()
    O.nw_batch(qp, qo[:ns], ql[:ns], rp, ro[:ns], rl[:ns], 2, -4, -4, -2, 32, threads=threads)
    tcn = time.perf_counter() - t0
    out["nw_1M_reads_band32"] = {
        "workload": "the 1,000,000 reads of the default SW workload against the 150 bp "
                    "reference window at their origin, banded NW, band 32, +2/-4/-4/-2",
        "scores_in_band": int((np.asarray(dev.nw_banded(dqn, drn, ncfg))["score"] > -900_000).sum()),
        "cells": ncells, "gpu_gcups": round(ncells / tnw / 1e6, 2), "gpu_ms": round(tnw, 3),
        "cpu_gcups": round(int((ql[:ns] * 65).sum()) / tcn / 1e9, 3), "cpu_cores": threads,
        "cpu_sample": f"first {ns} pairs",
    }
    dqn.close()
    drn.close()
    dq.close()
    dr.close()
    out["graph_replay"] = graph_bench(dev)
    out["serving"] = serve_bench(dev)
    return out


def graph_bench(dev, calls=200):
    """Per-call host time of small resident batches, eager (the default) vs replayed
    from a captured CUDA graph (GB2_FLAG_GRAPH): the first 2,000 pairs of the mixed-band SW
    workload (planning kernels and four class launches per call) and 5,000 reads of
    the default workload (one launch)."""
    from genomics_b200 import AlignConfig, synth
    from genomics_b200._lib import FLAG_GRAPH
    res = {}
    q3, r3, b3, _ = synth.generate(3, 2000)
    q1, r1, _, _ = synth.generate(1, 5000)
    for name, (q, r, bands) in (("mixed_sw_2000", (q3, r3, b3)), ("reads_5000", (q1, r1, None))):
        cfg = AlignConfig(*SCORING, 32)
        dq, dr = dev.upload_batch(q, with_nmask=False), dev.upload_batch(r, with_nmask=False)
        row = {}
        for mode, fl in (("eager_us", 0), ("graph_us", FLAG_GRAPH)):
            for _ in range(3):
                dev.sw_banded(dq, dr, cfg, bands=bands, flags=fl)
            dev.synchronize()
            t0 = time.perf_counter()
            for _ in range(calls):
                dev.sw_banded(dq, dr, cfg, bands=bands, flags=fl)
            row[mode] = round((time.perf_counter() - t0) / calls * 1e6, 1)
        res[name] = row
        dq.close()
        dr.close()
    return res


def _window_batch(batch, start, length, chunk=100_000):
    """Bases [start, start + length) of every sequence of an append-layout batch, as
    a new batch (2-bit MSB-first words, each sequence word-aligned)."""
    from genomics_b200 import SequenceBatch
    p, _, o, l = batch.arrays()
    n = o.size
    assert (l >= start + length).all()
    nw_in = int((int(l.max()) + 31) // 32)
    nw_out = (length + 31) // 32
    out = np.zeros(n * nw_out, np.uint64)
    shifts = (62 - 2 * np.arange(32, dtype=np.uint64)).astype(np.uint64)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        idx = o[c0:c1, None] + np.arange(nw_in)
        w = p[np.minimum(idx, p.size - 1)]
        bases = ((w[:, :, None] >> shifts) & np.uint64(3)).reshape(c1 - c0, -1)
        win = np.zeros((c1 - c0, nw_out * 32), np.uint64)
        win[:, :length] = bases[:, start:start + length]
        words = (win.reshape(c1 - c0, nw_out, 32) << shifts).sum(axis=2, dtype=np.uint64)
        out[c0 * nw_out:c1 * nw_out] = words.reshape(-1)
    offs = np.arange(n, dtype=np.int64) * nw_out
    return SequenceBatch.from_arrays(out, np.zeros_like(out), offs, np.full(n, length, np.int64))


def _slice(batch, i0, i1):
    """Pairs [i0, i1) of an append-layout SequenceBatch, without copying words."""
    from genomics_b200 import SequenceBatch
    p, m, o, l = batch.arrays()
    w0 = int(o[i0])
    w1 = int(o[i1 - 1] + (l[i1 - 1] + 31) // 32)
    return SequenceBatch.from_arrays(p[w0:w1], m[w0:w1], o[i0:i1] - w0, l[i0:i1])


def serve_bench(dev, pool_requests=320, pool_pairs=40_000):
    """Served mixed stream: Poisson arrivals of requests of 1-4,096 pairs (log-uniform),
    each pair SW (band 32/64/128) or WFA, 100-20,000 bp, divergence up to 15%.
    One pool of requests is drawn once.  The peak is the completion rate of the whole
    pool submitted at once; each load level then replays the same pool (the 0.2 level
    its first half) with Poisson arrivals at f x peak requests/s, so every offered
    fraction is relative to the capacity measured on the same work.  Latency = submit to
    results written, measured by the server."""
    from genomics_b200 import AlignConfig, WFAConfig, synth
    from genomics_b200.serve import AlignmentServer
    q, r, bands, kinds = synth.generate(4, pool_pairs)
    swc = AlignConfig(*SCORING, 32)
    wcfg = WFAConfig(4, 6, 2, synth.wfa_max_error_cover(q, r, 4, 6, 2))
    rng = np.random.default_rng(0xB2000004)
    n_req = pool_requests
    sizes = np.minimum(np.round(np.exp(rng.uniform(0, np.log(4096), n_req))).astype(int), 4096)
    starts = rng.integers(0, pool_pairs - 4096, n_req)

    def make(j):
        i0, i1 = int(starts[j]), int(starts[j] + sizes[j])
        return (_slice(q, i0, i1), _slice(r, i0, i1), bands[i0:i1], kinds[i0:i1])

    pool = [make(j) for j in range(n_req)]
    res = {"workload": "requests of 1-4,096 pairs (log-uniform), each pair SW (band 32/64/128) "
                       "or WFA (p=0.5), 100-20,000 bp log-uniform, divergence 0-15%",
           "max_error": int(wcfg.max_error), "pool_requests": n_req,
           "pool_pairs": int(sum(len(x[2]) for x in pool)),
           "method": "peak = completion rate of the pool submitted at once; each level "
                     "replays the same pool with Poisson arrivals at f x peak"}
    with AlignmentServer(dev, hbm_budget_bytes=32 << 30, max_inflight_groups=4) as srv:
        # warm the server's executors and buffers on a slice of the pool
        for pr in [srv.submit(a, b, swc, wcfg, kinds=k, bands=bd) for a, b, bd, k in pool[:16]]:
            pr.wait(600_000)
        t0 = time.perf_counter()
        prs = [srv.submit(a, b, swc, wcfg, kinds=k, bands=bd) for a, b, bd, k in pool]
        for pr in prs:
            pr.wait(600_000)
        t_peak = time.perf_counter() - t0
        peak = n_req / t_peak
        res["peak_requests_per_s"] = round(peak, 2)
        res["peak_pairs_per_s"] = round(res["pool_pairs"] / t_peak, 1)
        levels = []
        for f in (0.2, 0.4, 0.6, 0.8, 1.0):
            lam = f * peak
            batch = pool[:n_req // 2] if f < 0.3 else pool
            arrivals = np.cumsum(rng.exponential(1.0 / lam, len(batch)))
            prs = []
            tstart = time.perf_counter()
            for j, (a, b, bd, k) in enumerate(batch):
                delay = tstart + arrivals[j] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                prs.append(srv.submit(a, b, swc, wcfg, kinds=k, bands=bd))
            for pr in prs:
                pr.wait(600_000)
            t_all = time.perf_counter() - tstart
            lat = np.array([pr.latency_ms for pr in prs])
            levels.append({"offered_fraction": f, "offered_requests_per_s": round(lam, 2),
                           "requests": len(batch),
                           "pairs_per_s": round(sum(len(x[2]) for x in batch) / t_all, 1),
                           "p50_ms": round(float(np.percentile(lat, 50)), 2),
                           "p99_ms": round(float(np.percentile(lat, 99)), 2)})
        res["levels"] = levels
        res["p99_ms_at_0.8"] = next(l["p99_ms"] for l in levels if l["offered_fraction"] == 0.8)
        res["server"] = srv.stats()
    return res


def main():
    args = parse()
    if args.wfa_pass > 0:
        wfa_pass(args.wfa_pass)
        return
    dist = Dist()
    if args.impl == "reference":
        reference_arm(args, dist)
    else:
        our_arm(args, dist)


if __name__ == "__main__":
    main()
