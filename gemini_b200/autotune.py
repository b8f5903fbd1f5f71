"""Autotuner of the batched step's launch parameters, cached per instance-shape set.

The tunables do not change results (every instance computes the same bits whatever the
schedule); they change how the (instance, block) work items are laid onto the GPU:

* ``GRID_PCT``: persistent grid as a percentage of the occupancy limit, or 0 for one block
  per work item (the hardware block scheduler balances the items);
* ``DIFF_BLOCKS``: resident diffusion blocks per SM (each four warps, each warp solving 32
  columns): fewer blocks leave the SMs to the other phases' tails, more hide more latency.

``tune(batch)`` times each candidate with CUDA events over a few steps (after one warm-up
step, which also captures the graph) and keeps the fastest; results are cached in a JSON
file keyed by the sorted instance shapes (and the GPU name), so a later batch of the same
shapes starts from the cached choice.  Cache: $GEMINI_B200_CACHE or
~/.cache/gemini_b200/autotune.json.
"""
from __future__ import annotations

import hashlib
import json
import os

from . import batch as BT

CANDIDATES = [
    {BT.GRID_PCT: 0, BT.DIFF_BLOCKS: 4},
    {BT.GRID_PCT: 100, BT.DIFF_BLOCKS: 4},
    {BT.GRID_PCT: 200, BT.DIFF_BLOCKS: 4},
    {BT.GRID_PCT: 0, BT.DIFF_BLOCKS: 2},
    {BT.GRID_PCT: 0, BT.DIFF_BLOCKS: 3},
]


def cache_path() -> str:
    p = os.environ.get("GEMINI_B200_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "gemini_b200", "autotune.json")


def signature(batch: BT.Batch) -> str:
    import torch

    shapes = sorted((dg.grid.lx1, dg.grid.lx2, dg.grid.lx3, int(bool(dg.grid.unit_metrics)))
                    for dg, _, _ in batch.instances)
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    # "diff_blocks": the tunables' meaning (a cache written for other tunables does not apply)
    return hashlib.sha1(json.dumps(["diff_blocks", dev, shapes]).encode()).hexdigest()


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def apply(batch: BT.Batch, params: dict) -> None:
    for k, v in params.items():
        batch.set_param(int(k), int(v))


def time_steps(batch: BT.Batch, steps: int = 3) -> float:
    """Mean ms per batched step (one untimed warm-up step first)."""
    import torch

    batch.step()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        batch.step()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def tune(batch: BT.Batch, steps: int = 3, use_cache: bool = True, candidates=None) -> dict:
    """Pick the fastest candidate for this batch (advances its state by the timed steps).
    Returns {"params": ..., "ms_per_step": ..., "trials": [...], "cached": bool}."""
    sig = signature(batch)
    cache = _load() if use_cache else {}
    if use_cache and sig in cache:
        params = {int(k): v for k, v in cache[sig]["params"].items()}
        apply(batch, params)
        return {"params": params, "ms_per_step": cache[sig]["ms_per_step"], "trials": [], "cached": True}
    trials = []
    for cand in (candidates or CANDIDATES):
        apply(batch, cand)
        trials.append((time_steps(batch, steps), cand))
    best_ms, best = min(trials, key=lambda t: t[0])
    apply(batch, best)
    if use_cache:
        cache[sig] = {"params": {str(k): v for k, v in best.items()}, "ms_per_step": best_ms}
        _store(cache)
    return {"params": best, "ms_per_step": best_ms,
            "trials": [{"params": c, "ms_per_step": t} for t, c in trials], "cached": False}
