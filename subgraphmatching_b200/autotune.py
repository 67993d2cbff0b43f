"""Autotuner for the enumeration launch (no counterpart in the reference).

Times a small grid of launch and intersection settings — warps per block,
task grab, staged chunk, galloping ratio, last-depth bitmap threshold,
register-capped build — on a sample of the caller's queries through the
batched entry point (one persistent launch under a CUDA graph), keeps the
fastest, and writes the choice with its timings to a JSON file that
`load` reads back.  Settings never change counts; the tuner checks that
every setting returns the same counts as the first.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import asdict

from . import EnumOptions, explore_batch

GRID = [
    dict(),
    dict(warps_per_block=4),
    dict(task_grab=1),
    dict(task_grab=16),
    dict(stage_chunk=2048),
    dict(stage_chunk=512),
    dict(gallop_ratio=4),
    dict(gallop_ratio=64),
    dict(bitmap_min=8),
    dict(bitmap_min=256),
    dict(bitmap_min=-1),
    dict(blocks_per_sm=3),
]

# the cache + failing-set explorer has no last-depth bitmap
GRID_CACHE = [g for g in GRID if "bitmap_min" not in g]


def autotune(graph, queries, cans, orders=None, cap: int = 0, budget_ms: float = 0.0, explore: int = 0,
             grid=None, repeats: int = 2, path: str | None = None) -> tuple[EnumOptions, dict]:
    """Returns (best options, report); writes the report to `path` if given."""
    grid = GRID if grid is None else grid
    report = {"queries": len(queries), "cap": cap, "budget_ms": budget_ms, "explore": explore, "trials": []}
    best, best_ms, ref_counts = None, float("inf"), None
    for setting in grid:
        opts = EnumOptions(explore=explore, time_budget_ms=budget_ms, budget_per_query=1, **setting)
        times = []
        for _ in range(repeats):
            counts, st = explore_batch(graph, queries, cans, orders, opts, cap)
            times.append(st.kernel_ms)
        timed_out = st.status != 0
        if not timed_out:
            if ref_counts is None:
                ref_counts = counts
            elif counts != ref_counts:
                raise AssertionError(f"setting {setting} changed the counts")
        else:  # queries at the budget are partial; the setting is still ranked by its time
            timed_out = False
        ms = min(times)
        report["trials"].append({"setting": setting, "kernel_ms": ms, "timed_out": timed_out})
        if not timed_out and ms < best_ms:
            best, best_ms = opts, ms
    best = best or EnumOptions(explore=explore)
    best.time_budget_ms = 0.0
    best.budget_per_query = 0
    report["best"] = asdict(best)
    report["best_kernel_ms"] = best_ms
    report["when"] = time.strftime("%Y-%m-%dT%H:%M:%S")
    if path:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path, "w") as f:
            json.dump(report, f, indent=1)
    return best, report


def load(path: str) -> EnumOptions:
    """The options an earlier autotune run chose."""
    with open(path) as f:
        return EnumOptions(**json.load(f)["best"])
