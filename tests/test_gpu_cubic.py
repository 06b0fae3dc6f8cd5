"""The cubic shape extension (AGPU_SHAPE_CUBIC) on the device against the
oracle's FP64 restatement of it.  The reference has no cubic gather or
deposit; the oracle's cubic Esirkepov deposit is pinned by the discrete
continuity test of tests/test_oracle.py.

* FP64 form, deterministic mode: particles, fields and currents bit-exact
  against the oracle after 24 steps with window shifts, injection and
  removal.
* FP64 form with atomics: fields within 1e-9 after 24 steps.
* FP32 split form: relative L2 field error <= 1e-3 against the FP64 oracle
  after 40 steps.
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64, AGPU_SHAPE_CUBIC, AgpuError
from aladyn_b200.sim import PicDevice
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case, sort_records

pytestmark = pytest.mark.gpu


def _pair(ndim, precision=AGPU_FP64):
    p = small_case(ndim, precision=precision)
    p.shape = AGPU_SHAPE_CUBIC
    p_o = small_case(ndim, precision=AGPU_FP64)
    p_o.shape = AGPU_SHAPE_CUBIC
    dev, ora = PicDevice(p), Oracle(p_o)
    ebf = laser_fields(p)
    src = plasma_source(p)
    for s in (dev, ora):
        s.set_fields(ebf)
        s.set_plasma_source(src)
        s.load_plasma(0)
    return p, dev, ora


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ndim", [2, 3])
def test_cubic_fp64_deterministic_bitexact(ndim):
    p, dev, ora = _pair(ndim)
    dev.set_deterministic(True)
    t = 0.0
    for it in range(24):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0 and ora.error_bits() == 0
        assert out.np[0] == oo.np[0], (it, out.np[0], oo.np[0])
        t += p.dt
    a, b = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert np.array_equal(dev.get_fields().view(np.uint64), ora.get_fields().view(np.uint64))


@pytest.mark.parametrize("ndim", [2, 3])
def test_cubic_fp64_atomic_close(ndim):
    p, dev, ora = _pair(ndim)
    t = 0.0
    for it in range(24):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert out.np[0] == oo.np[0]
        t += p.dt
    assert _relmax(dev.get_fields(), ora.get_fields()) <= 1e-9
    a, b = sort_records(dev.get_species(0)), sort_records(ora.get_species(0))
    assert a.shape == b.shape
    assert np.abs(a[:, :ndim] - b[:, :ndim]).max() <= 1e-9


@pytest.mark.parametrize("ndim", [2, 3])
def test_cubic_fp32_split_vs_fp64(ndim):
    p, dev, ora = _pair(ndim, precision=AGPU_FP32_SPLIT)
    t = 0.0
    for it in range(40):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert out.error_bits == 0
        t += p.dt
    fa, fb = dev.get_fields(), ora.get_fields()
    sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2) if ndim == 3 else slice(0, 1))
    for c in range(p.nfield):
        a, b = fa[sl + (c,)], fb[sl + (c,)]
        nb = np.linalg.norm(b)
        if nb > 0:
            assert np.linalg.norm(a - b) / nb <= 1e-3, (c, np.linalg.norm(a - b) / nb)
    assert abs(out.np[0] - oo.np[0]) <= max(2, 1e-4 * oo.np[0])


def test_cubic_shapes_differ_from_quadratic():
    """The shape switch changes the physics (a run with cubic shapes is not
    the quadratic run), and the split form refuses the per-particle
    deterministic mode, which has the quadratic shapes only."""
    p, dev, ora = _pair(3)
    q = small_case(3)
    dq = PicDevice(q)
    dq.set_fields(laser_fields(q))
    dq.set_plasma_source(plasma_source(q))
    dq.load_plasma(0)
    t = 0.0
    for it in range(5):
        dev.lp_run(t, it, initial_time=(it == 0))
        dq.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    assert _relmax(dev.get_fields(), dq.get_fields()) > 1e-6
    p32 = small_case(3, precision=AGPU_FP32_SPLIT)
    p32.shape = AGPU_SHAPE_CUBIC
    d32 = PicDevice(p32)
    with pytest.raises(AgpuError):
        d32.set_deterministic(True)
