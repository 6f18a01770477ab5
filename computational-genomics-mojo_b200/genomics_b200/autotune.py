"""Autotuner of the batched alignment kernels (gb2_autotune).

The Smith-Waterman int32 register kernels split a band row over G lanes of K
columns each, and the WFA kernel takes 4, 2 or 1 diagonals per thread per round
at 3-5 resident blocks per SM; every shape computes the same results.  `tune`
times each shape on a sample of the caller's own pairs, installs the fastest
in the device's context, and returns the table; `save` / `load` keep it in a
JSON file so a service tunes once per machine and restores the table at
start-up.
"""
from __future__ import annotations

import json

SW_BANDS = (16, 32, 64, 128)


def tune(device, q, r, sw_cfg=None, wfa_cfg=None, bands=SW_BANDS, n_pairs=None, reps=5,
         pair_bands=None):
    """Tunes the SW register kernel of every band class in `bands` (with sw_cfg's
    scores) and, given wfa_cfg, the WFA kernel, on resident batches q, r.  With
    `pair_bands` (the batch's per-pair bands) each class is tuned inside the whole
    mixed call, one class after another.  Tune on the batch size that will run.
    Returns {"sw": {band: variant}, "wfa": variant, "measurements": {...}}."""
    from dataclasses import replace
    table = {"sw": {}, "wfa": None, "measurements": {}}
    if sw_cfg is not None:
        for b in bands:
            res = device.autotune("sw", q, r, replace(sw_cfg, band_width=int(b)), n_pairs, reps,
                                  bands=pair_bands)
            table["sw"][str(b)] = res["chosen"]
            table["measurements"][f"sw_{b}"] = res["candidates"]
    if wfa_cfg is not None:
        res = device.autotune("wfa", q, r, wfa_cfg, n_pairs, reps)
        table["wfa"] = res["chosen"]
        table["measurements"]["wfa"] = res["candidates"]
    return table


def install(device, table):
    """Installs a table returned by `tune` (or read by `load`) into the context."""
    for b, v in table.get("sw", {}).items():
        device.tune_set("sw", int(v), int(b))
    if table.get("wfa") is not None:
        device.tune_set("wfa", int(table["wfa"]))


def save(table, path):
    with open(path, "w") as f:
        json.dump(table, f, indent=1)


def load(device, path):
    with open(path) as f:
        table = json.load(f)
    install(device, table)
    return table
