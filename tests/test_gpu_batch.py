"""Batched instances (agpu_batch_*) and the deferred-count mode.

* Deferred counts (with and without CUDA-graph replay of the steps between
  window shifts): one instance stepped with the per-step host
  synchronisation and a copy stepped in deferred mode agree (FP64 form,
  25 steps across two window shifts): particle counts equal, fields within
  1e-9 (only the atomic summation order of the deposit differs).
* A batch of 2D instances of different sizes, lasers and densities advanced
  by agpu_batch_run (multi-instance steps between window shifts, or every
  instance on its own stream) against the same instances run one after the
  other through agpu_step: counts and pushes equal, fields within 1e-9
  (FP64) or 1e-4 relative L2 (FP32 split, where atomic order changes the
  roundings).
"""
import math

import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.config import Grid, laser, make_params, n_over_nc_to_n0, plasma
from aladyn_b200.sim import PicBatch, PicDevice

pytestmark = pytest.mark.gpu
LAM0 = 0.8


def scan_instance(i, precision, nx=None, ny=None):
    """A small 2D LWFA instance (dx = 0.05 lambda, dy = 0.2 lambda, 4 ppc)."""
    sizes = [(64, 32), (96, 32), (128, 48), (80, 64), (64, 40), (112, 32)]
    nx = nx or sizes[i % len(sizes)][0]
    ny = ny or sizes[i % len(sizes)][1]
    g = Grid(2, nx, ny, 1, k0=25.0, yx_rat=4.0, zx_rat=1.0, cfl=0.8)
    cap = nx * ny * 4 * 2 + 4096
    p = make_params(g, precision=precision, capacity=(cap, 0, 0, 0), w_sh=10, w_speed=1.0)
    lx = nx * p.dx
    a0 = 1.0 + 0.4 * i
    las = laser(a0, LAM0, (2.0 + 0.2 * i) * LAM0, 0.25 * lx, xc=0.6 * lx, xf=0.6 * lx)
    n0 = n_over_nc_to_n0(0.01 * (1 + 0.1 * i), LAM0)
    src = plasma(0, 2, 2, 1, -1, n0 / 4, x_start=p.gxmin + 0.2 * lx, x_end=1.0e7, y_min=p.gymin,
                 y_max=p.gymax, jitter=0.5, seed=1000 + i)
    return p, las, src


def _setup(dev, las, src):
    dev.init_laser(las)
    dev.set_plasma_source(src)
    dev.load_plasma(0)


def _run_sync(p, las, src, steps, deferred=False, graphs=False):
    dev = PicDevice(p)
    _setup(dev, las, src)
    if deferred:
        dev.set_deferred_counts(True)
        dev.set_step_graphs(graphs)
    t = 0.0
    for it in range(steps):
        dev.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    dev.synchronize()
    return dev


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("graphs", [False, True])
def test_deferred_counts_match_synchronous_steps(graphs):
    """Deferred counts, with or without the step graphs replaying the steps
    between window shifts, against per-step synchronous steps."""
    p, las, src = scan_instance(2, AGPU_FP64)
    a = _run_sync(p, las, src, 25)
    b = _run_sync(p, las, src, 25, deferred=True, graphs=graphs)
    assert a.count(0) == b.count(0) > 0
    assert a.timers().pushes == b.timers().pushes
    assert _rel(b.get_fields(), a.get_fields()) < 1e-9


@pytest.mark.parametrize("precision,multi", [(AGPU_FP64, True), (AGPU_FP32_SPLIT, True), (AGPU_FP32_SPLIT, False)])
def test_batch_matches_sequential_instances(precision, multi):
    """multi: the steps between window shifts run as one multi-instance step
    (split form; FP64 instances step one by one either way)."""
    n, steps = 6, 25
    cases = [scan_instance(i, precision) for i in range(n)]
    batch = PicBatch([c[0] for c in cases])
    batch.set_multi(multi)
    for d, (p, las, src) in zip(batch.instances, cases):
        _setup(d, las, src)
    status = batch.run(steps, nthreads=3)
    assert status == [0] * n
    if multi and precision == AGPU_FP32_SPLIT:
        assert batch.launches() > 0  # the multi-instance path ran
    for i, (p, las, src) in enumerate(cases):
        it, t = batch.clock(i)
        assert it == steps and abs(t - steps * p.dt) < 1e-9
        ref = _run_sync(p, las, src, steps)
        got = batch.instances[i]
        if precision == AGPU_FP64:
            assert got.count(0) == ref.count(0)
            assert got.timers().pushes == ref.timers().pushes
            assert _rel(got.get_fields(), ref.get_fields()) < 1e-9
        else:
            assert abs(got.count(0) - ref.count(0)) <= 2
            fa, fb = got.get_fields(), ref.get_fields()
            l2 = math.sqrt(((fa - fb) ** 2).sum() / (fb ** 2).sum())
            assert l2 < 1e-4
        ref.close()
    batch.close()
