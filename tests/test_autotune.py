"""The run-option tuner (aladyn_b200/autotune.py) on CPU: candidate
enumeration, the choice of the fastest measured candidate, failed
candidates never chosen, and the JSON cache keyed by the workload."""
import math

import pytest

from aladyn_b200.autotune import (BATCH_SPACE, STEP_SPACE, Tuner, apply_step_options, candidates, workload_key)
from aladyn_b200.config import Grid, make_params


def _p(ndim=2, nx=64, ny=32, nz=16):
    g = Grid(ndim, nx, ny, nz if ndim == 3 else 1, k0=25.0, yx_rat=4.0, zx_rat=4.0, cfl=0.8)
    return make_params(g)


def test_candidates_cover_the_space():
    c = candidates(STEP_SPACE)
    assert len(c) == math.prod(len(v) for v in STEP_SPACE.values())
    assert len({tuple(sorted(d.items())) for d in c}) == len(c)
    pinned = candidates(STEP_SPACE, fixed={"graphs": True})
    assert all(d["graphs"] for d in pinned) and len(pinned) == len(c) // 2
    assert len(candidates(BATCH_SPACE)) == 6


def test_workload_key():
    a, b = _p(2), _p(3)
    assert workload_key(a, 4) != workload_key(b, 4)
    assert workload_key(a, 4) != workload_key(a, 8)
    assert workload_key(a, 4, 256) != workload_key(a, 4, 1)
    assert workload_key(a, 4) == workload_key(_p(2), 4)


def test_tuner_picks_fastest_and_caches(tmp_path):
    path = str(tmp_path / "tune.json")
    calls = []

    def measure(o):
        calls.append(o)
        if o["sort_interval"] == 16:
            raise RuntimeError("does not run")
        return 10.0 - 3.0 * o["fused_yee"] - 2.0 * o["graphs"] + 0.1 * o["sort_interval"]

    t = Tuner(path)
    r = t.tune("k1", STEP_SPACE, measure)
    assert r.best == {"fused_yee": True, "graphs": True, "sort_interval": 0}
    assert r.ms_per_step == pytest.approx(5.0)
    assert not r.cached and len(r.tried) == len(candidates(STEP_SPACE))
    assert all(ms == math.inf for o, ms in r.tried if o["sort_interval"] == 16)
    n = len(calls)
    # a second tuner reads the cache and measures nothing
    r2 = Tuner(path).tune("k1", STEP_SPACE, measure)
    assert r2.cached and r2.best == r.best and len(calls) == n
    # force measures again
    r3 = Tuner(path).tune("k1", STEP_SPACE, measure, force=True)
    assert not r3.cached and len(calls) == 2 * n
    assert r3.as_dict()["tried"][0]["options"] in candidates(STEP_SPACE)


def test_tuner_refuses_when_nothing_runs(tmp_path):
    def measure(o):
        raise RuntimeError("no")

    with pytest.raises(RuntimeError):
        Tuner(str(tmp_path / "t.json")).tune("k", BATCH_SPACE, measure)


def test_apply_step_options():
    class Dev:
        def __init__(self):
            self.log = []

        def set_sort_interval(self, n):
            self.log.append(("sort", n))

        def set_fused_yee(self, on):
            self.log.append(("fused", on))

        def set_deferred_counts(self, on):
            self.log.append(("defer", on))

        def set_step_graphs(self, on):
            self.log.append(("graphs", on))

    d = Dev()
    apply_step_options(d, {"sort_interval": 8, "fused_yee": True, "graphs": True})
    assert d.log == [("sort", 8), ("fused", True), ("defer", True), ("graphs", True)]
    d = Dev()
    apply_step_options(d, {"sort_interval": 0, "fused_yee": False, "graphs": False})
    assert ("graphs", True) not in d.log and ("defer", True) not in d.log
