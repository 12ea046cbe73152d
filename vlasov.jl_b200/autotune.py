"""Autotuner of the launch shapes of one run (vlb_set_tuning).

The shapes are the gather's form (its sums over y on the tensor cores or
on the FP32 pipes), the particles per work item of the gather and the coarse
deposit (`chunk`) and the CTAs per SM of the persistent grids of the gather,
the coarse deposit, the push and the record move of the sort.  They change
no result beyond the order of float32 atomic sums, only the time.

The tuner works on the run as it is: it snapshots the cloud and the
projectile, times candidate shapes on real steps (eager, with the library's
per-stage events, so that each shape is judged by the stages it touches),
and restores the snapshot.  Coordinate descent: `chunk` first (it moves the
work items of both the gather and the coarse deposit), then each grid size
on its own stage.  Results can be kept in a JSON cache keyed by the GPU, the
grid and the cloud size.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

# candidate values, and the stages each shape is judged by
SEARCH = {
    "field_tensor_cores": ((1, 0), ("forces",)),
    "chunk": ((64, 128, 256), ("deposit_coarse", "forces", "sort")),
    "field_ctas_per_sm": ((2, 3, 4), ("forces",)),
    "cic_ctas_per_sm": ((2, 4, 8), ("deposit_coarse",)),
    "push_ctas_per_sm": ((2, 4, 8), ("push",)),
    "move_ctas_per_sm": ((2, 4, 8), ("sort",)),
}


def _stage_ms(sim, steps: int) -> dict:
    acc = sim.accelerator
    use_graph = sim.use_graph
    sim.use_graph = False
    acc.profile(True)
    try:
        for _ in range(steps):
            sim.step()
        return {k: v / steps for k, v in acc.stage_times().items()}
    finally:
        acc.profile(False)
        sim.use_graph = use_graph


def tune(sim, *, steps: int = 3, warmup: int = 1, search=None) -> dict:
    """Best launch shapes for `sim` (a Simulation), left set on its context;
    the cloud and the projectile are restored as they were."""
    search = SEARCH if search is None else search
    acc = sim.accelerator
    snap = sim.snapshot()
    best = acc.tuning()
    try:
        for name, (values, stages) in search.items():
            times = {}
            for v in values:
                acc.set_tuning(**{**best, name: v})
                sim.restore(snap)
                for _ in range(warmup):
                    sim.step()
                sim.restore(snap)
                st = _stage_ms(sim, steps)
                times[v] = sum(st[s] for s in stages)
            best[name] = min(times, key=times.get)
        acc.set_tuning(**best)
    finally:
        sim.restore(snap)
    return best


def cache_key(sim) -> str:
    import torch
    name = torch.cuda.get_device_name(sim.accelerator.device) if torch.cuda.is_available() else "cpu"
    n = sim.meshes.fine.n
    npart = sim.params.nparticles
    bucket = 1 << max(0, (int(npart) - 1).bit_length())  # the next power of two
    return f"{name}|n={n}|npart<={bucket}"


def tune_cached(sim, path: str | os.PathLike | None, **kw) -> dict:
    """tune(), through a JSON cache file at `path` (None: no cache)."""
    if path is None:
        return tune(sim, **kw)
    path = Path(path)
    cache = json.loads(path.read_text()) if path.exists() else {}
    key = cache_key(sim)
    if key in cache:
        sim.accelerator.set_tuning(**cache[key])
        return cache[key]
    best = tune(sim, **kw)
    cache[key] = best
    path.write_text(json.dumps(cache, indent=1, sort_keys=True))
    return best
