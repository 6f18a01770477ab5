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
  roofline    integer-ALU view of the dominant kernel: cells x 11 int32 ops (the
              reference recurrence as written) against the lane-op peak measured by
              the library's own microkernels in the same run; an HBM view beside it.
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
    ap.add_argument("--no-peaks", action="store_true", help="skip the integer-throughput probes")
    ap.add_argument("--variant", type=int, default=0, help="kernel variant knob (tuning)")
    ap.add_argument("--plain", action="store_true", help="plain launch instead of the queue")
    return ap.parse_args()


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


def reference_arm(args, dist: Dist):
    """The reference's CPU algorithm, timed on this host's cores."""
    if dist.rank != 0:
        dist.close()
        return
    from genomics_b200 import synth
    threads = os.cpu_count() or 1
    q, r, _, _ = synth.generate(1, args.pairs)
    sample = min(args.pairs, max(1000, args.cpu_sample // 2))
    for _ in range(args.warmup):
        cpu_sw_gcups(q, r, min(sample, 5000), threads)
    times, cells = [], 0
    ql = q.arrays()[3]
    per_step_cells = int((ql[:sample] * (2 * BAND + 1)).sum())
    for _ in range(args.steps):
        _, n, dt = cpu_sw_gcups(q, r, sample, threads)
        times.append(dt)
        cells += per_step_cells
    total = sum(times)
    value = cells / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GCUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step": sample,
                   "note": "reference is Mojo-only (no toolchain here); its CPU algorithm "
                           "runs as the C restatement in oracle/"},
        "cpu_baseline": {"value": round(value, 4), "unit": "GCUPS", "cores": threads,
                         "kind": "port",
                         "sample": f"{sample} of the {args.pairs} pairs per step"},
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
    h2d = sum(a.nbytes for a in (q.packed, q.offsets, q.lengths, r.packed, r.offsets, r.lengths))
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
        achieved_ops = kern_gcups * SW_OPS_PER_CELL
        alg_bytes = h2d - 0 + d2h  # packed words + metadata read, results written
        mp = {}
        mp_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(mp_path):
            mp = json.load(open(mp_path))
        hbm_peak = mp.get("hbm_gbs", 6650.0)
        cpu = None
        if args.gpus == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            g, n, dt = cpu_sw_gcups(q, r, args.cpu_sample, threads)
            cpu = {"value": round(g, 4), "unit": "GCUPS", "cores": threads, "kind": "port",
                   "sample": f"first {n} pairs of the workload ({dt:.1f} s)"}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GCUPS",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "pairs_per_gpu": args.pairs, "band": BAND,
                       "query_bp": 150, "target_bp": 200, "scoring": list(SCORING),
                       "path": "batched" if batched else "plain", "variant": args.variant,
                       "l2": "flushed between timed steps (256 MB device write)",
                       "cells_per_step_per_gpu": cells},
            "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "GCUPS",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "roofline": {"bound": "int_alu", "achieved": round(achieved_ops, 1),
                         "peak": peak_ops, "unit": "Gop/s",
                         "frac": round(achieved_ops / peak_ops, 4),
                         "ops_per_cell": SW_OPS_PER_CELL,
                         "kernel_ms": round(kernel_ms, 4),
                         "kernel_gcups": round(kern_gcups, 2),
                         "peak_source": "gb2_int_peak microkernels in this run: "
                                        "max(IADD, IMNMX, 2 x DPX viaddmax) lane-ops/s",
                         "traffic": None,
                         "hbm": {"achieved": round(alg_bytes / (kernel_ms * 1e-3) / 1e9, 2),
                                 "peak": hbm_peak, "unit": "GB/s",
                                 "frac": round(alg_bytes / (kernel_ms * 1e-3) / 1e9 / hbm_peak, 5),
                                 "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}},
            "int_peaks_gops": peaks,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
    dq.close()
    dr.close()
    dev.close()
    dist.close()
    if line:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    dist = Dist()
    if args.impl == "reference":
        reference_arm(args, dist)
    else:
        our_arm(args, dist)


if __name__ == "__main__":
    main()
