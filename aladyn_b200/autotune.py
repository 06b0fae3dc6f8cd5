"""Autotuning of the run options that have no single best value.

The library leaves a few choices to the caller because the best one depends
on the grid, the particle count and the GPU: the sort interval (how often
the records move in memory along the tile order), the fused Yee kernel
(faster on small 2D grids, slower in 3D), step graphs (they remove the
per-kernel launch cost, which only matters on small grids) and, for batched
parameter scans, the worker threads that queue the instances' special steps
and the sort interval of the instances.  The tuner runs each candidate for a
few steps on a fresh instance built by the caller, times the steps with CUDA
events on the launching stream, keeps the fastest and caches the choice in
a JSON file keyed by the workload (dimension, grid, particles per cell,
precision, shape, instance count), so that later runs of the same workload
reuse it without measuring again.

The reference has no counterpart: its run options are namelist inputs.
"""
from __future__ import annotations

import itertools
import json
import os
from dataclasses import dataclass, field

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "aladyn_b200", "tune.json")

# candidate values of the options the tuner may set
STEP_SPACE = {"sort_interval": (0, 8, 16), "fused_yee": (False, True), "graphs": (False, True)}
BATCH_SPACE = {"threads": (8, 16, 32), "sort_interval": (0, 8)}


def workload_key(p, ppc: int, instances: int = 1) -> str:
    """Cache key of a workload: dimension, grid, particles per cell,
    precision, shape and, for batches, the instance count (the first
    instance's grid)."""
    nz = p.nz if p.ndim == 3 else 1
    return f"{p.ndim}d:{p.nx}x{p.ny}x{nz}:ppc{ppc}:prec{p.precision}:shape{p.shape}:n{instances}"


def candidates(space: dict, fixed: dict | None = None):
    """Every combination of the space's values (fixed options pinned)."""
    fixed = fixed or {}
    keys = sorted(space)
    vals = [(fixed[k],) if k in fixed else space[k] for k in keys]
    return [dict(zip(keys, combo)) for combo in itertools.product(*vals)]


@dataclass
class TuneResult:
    key: str
    best: dict
    ms_per_step: float
    tried: list = field(default_factory=list)  # (options, ms per step)
    cached: bool = False

    def as_dict(self):
        return {"key": self.key, "best": self.best, "ms_per_step": self.ms_per_step, "cached": self.cached,
                "tried": [{"options": o, "ms_per_step": m} for o, m in self.tried]}


class Tuner:
    """Measure candidates with a caller-supplied function and cache the
    fastest.  ``measure(options) -> ms per step`` builds a fresh instance,
    applies the options, runs warm-up and timed steps and returns the device
    time per step (inf when the candidate failed)."""

    def __init__(self, cache_path: str | None = DEFAULT_CACHE):
        self.path = cache_path
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            try:
                with open(cache_path) as f:
                    self.cache = json.load(f)
            except (OSError, ValueError):
                self.cache = {}

    def lookup(self, key: str):
        e = self.cache.get(key)
        if e is None:
            return None
        return TuneResult(key, e["best"], e["ms_per_step"], [], cached=True)

    def store(self, r: TuneResult):
        self.cache[r.key] = {"best": r.best, "ms_per_step": r.ms_per_step}
        if not self.path:
            return
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def tune(self, key: str, space: dict, measure, fixed: dict | None = None, force: bool = False) -> TuneResult:
        if not force:
            r = self.lookup(key)
            if r is not None:
                return r
        tried = []
        for opts in candidates(space, fixed):
            try:
                ms = float(measure(opts))
            except Exception:  # a candidate that cannot run is never chosen
                ms = float("inf")
            tried.append((opts, ms))
        best, ms = min(tried, key=lambda t: t[1])
        if ms == float("inf"):
            raise RuntimeError(f"no candidate of {key} ran")
        r = TuneResult(key, best, ms, tried)
        self.store(r)
        return r


# ---- applying options ------------------------------------------------------------
def apply_step_options(dev, opts: dict):
    """Set a single instance's options (graphs need deferred counts)."""
    dev.set_sort_interval(int(opts.get("sort_interval", 0)))
    dev.set_fused_yee(bool(opts.get("fused_yee", False)))
    if opts.get("graphs", False):
        dev.set_deferred_counts(True)
        dev.set_step_graphs(True)


def apply_batch_options(batch, opts: dict):
    for d in batch.instances:
        d.set_sort_interval(int(opts.get("sort_interval", 0)))


def time_steps(torch, dev, p, warmup: int, steps: int) -> float:
    """ms per step of `steps` steps after `warmup` (CUDA events on the
    handle's stream)."""
    t, it = 0.0, 0
    for _ in range(warmup):
        dev.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
        it += 1
    s = torch.cuda.ExternalStream(dev.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev.synchronize()
    e0.record(s)
    for _ in range(steps):
        dev.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
        it += 1
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def tune_single(torch, make, p, ppc: int, warmup: int = 3, steps: int = 10, space: dict | None = None,
                tuner: Tuner | None = None, force: bool = False) -> TuneResult:
    """Tune a single-instance workload; ``make()`` returns a fresh, loaded
    PicDevice."""
    tuner = tuner or Tuner()

    def measure(opts):
        dev = make()
        try:
            apply_step_options(dev, opts)
            return time_steps(torch, dev, p, warmup, steps)
        finally:
            dev.close()

    return tuner.tune(workload_key(p, ppc), space or STEP_SPACE, measure, force=force)


def tune_batch(torch, make_batch, p0, ppc: int, n: int, warmup: int = 3, steps: int = 5, space: dict | None = None,
               tuner: Tuner | None = None, force: bool = False) -> TuneResult:
    """Tune a batched scan; ``make_batch()`` returns a fresh, loaded
    PicBatch of n instances."""
    tuner = tuner or Tuner()

    def measure(opts):
        b = make_batch()
        try:
            apply_batch_options(b, opts)
            st = b.run(warmup, int(opts["threads"]))
            if any(st):
                return float("inf")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            st = b.run(steps, int(opts["threads"]))
            e1.record()
            e1.synchronize()
            if any(st):
                return float("inf")
            return e0.elapsed_time(e1) / steps
        finally:
            b.close()

    return tuner.tune(workload_key(p0, ppc, n), space or BATCH_SPACE, measure, force=force)


__all__ = ["Tuner", "TuneResult", "STEP_SPACE", "BATCH_SPACE", "candidates", "workload_key", "apply_step_options",
           "apply_batch_options", "time_steps", "tune_single", "tune_batch", "DEFAULT_CACHE"]
