"""The fused z-streaming Yee step (agpu_set_fused_yee) against the six
separate sweeps and face kernels.

* FP64, deterministic deposit: the whole field array (interior, Mur faces and
  every ghost layer) bit-identical after 24 steps with window shifts, in 2D
  and 3D, on a grid whose size is not a multiple of the kernel's tile.
* FP32 split: within 1e-6 of the separate kernels (the two compile to
  different FP32 contractions).
* A vacuum pulse with random values in every ghost layer: one step, FP64,
  bit-identical over the whole array.
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.sim import PicDevice
from tests.helpers import laser_fields, plasma_source, small_case

pytestmark = pytest.mark.gpu


def _dev(ndim, precision, fused, **kw):
    p = small_case(ndim, precision=precision, **kw)
    d = PicDevice(p)
    d.set_fields(laser_fields(p))
    d.set_plasma_source(plasma_source(p))
    d.load_plasma(0)
    d.set_fused_yee(fused)
    return p, d


@pytest.mark.parametrize("ndim,dims", [(2, (70, 37, 1)), (3, (70, 37, 19))])
def test_fused_yee_fp64_bitexact(ndim, dims):
    kw = dict(nx=dims[0], ny=dims[1], nz=dims[2], cap=600_000)
    p, a = _dev(ndim, AGPU_FP64, False, **kw)
    _, b = _dev(ndim, AGPU_FP64, True, **kw)
    a.set_deterministic(True)
    b.set_deterministic(True)
    t = 0.0
    for it in range(24):
        oa = a.lp_run(t, it, initial_time=(it == 0))
        ob = b.lp_run(t, it, initial_time=(it == 0))
        assert oa.np[0] == ob.np[0]
        t += p.dt
    fa, fb = a.get_fields(), b.get_fields()
    assert np.array_equal(fa.view(np.uint64), fb.view(np.uint64))


@pytest.mark.parametrize("ndim", [2, 3])
def test_fused_yee_fp32_close(ndim):
    p, a = _dev(ndim, AGPU_FP32_SPLIT, False)
    _, b = _dev(ndim, AGPU_FP32_SPLIT, True)
    t = 0.0
    for it in range(12):
        a.lp_run(t, it, initial_time=(it == 0))
        b.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    fa, fb = a.get_fields(), b.get_fields()
    for c in range(p.nfield):
        sc = max(np.abs(fa[..., c]).max(), 1e-30)
        assert np.abs(fa[..., c] - fb[..., c]).max() <= 1e-4 * sc, c


@pytest.mark.parametrize("ndim", [2, 3])
def test_fused_yee_vacuum_random_ghosts(ndim):
    kw = dict(nx=45, ny=21, nz=13)
    p = small_case(ndim, precision=AGPU_FP64, **kw)
    rng = np.random.default_rng(11)
    ebf = laser_fields(p) + rng.standard_normal(laser_fields(p).shape) * 1e-3
    out = []
    for fused in (False, True):
        d = PicDevice(p)
        d.set_fields(np.asfortranarray(ebf))
        d.set_fused_yee(fused)
        d.lp_run(0.0, 1)  # no particles: field_bd, fold of zero currents, Yee; no window at iter 1
        out.append(d.get_fields())
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))
