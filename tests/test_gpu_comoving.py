"""The comoving frame (w_speed < 0) on the device against the oracle: the
pushers' x -= dt vbeam, the x advection substeps of the Yee step
(field_xadvect, src/fields/grid_fields.f90:210-324), comoving_coordinate's
removal and injection (src/dynamics/window.f90:227-275) and, in the
envelope cycle, env_lpf_solve with ib = 0 (grid_fields.f90:696-858).

Tolerances: deterministic mode bit-exact (particles, currents, fields,
env, the source scratch) over 16 steps with four coordinate shifts; atomic
sums: particles bit-exact after one step, currents and fields to 1e-12 of
their largest value."""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64, AgpuError
from aladyn_b200.sim import PicDevice
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case
from tests.test_envelope import env_case, numpy_init, pulse

pytestmark = pytest.mark.gpu

VB = 0.98


def _pair(ndim, w_sh=4):
    p = small_case(ndim, w_sh=w_sh)
    p.w_speed = -VB
    dev = PicDevice(p)
    ora = Oracle(p)
    ebf = 0.5 * laser_fields(p)
    dev.set_fields(ebf)
    ora.set_fields(ebf)
    src = plasma_source(p, x_start_frac=0.7)
    dev.set_plasma_source(src)
    ora.set_plasma_source(src)
    dev.load_plasma(0)
    ora.load_plasma(0)
    return p, dev, ora


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ndim", [2, 3])
def test_comoving_step_deterministic_bitexact(ndim):
    p, dev, ora = _pair(ndim)
    dev.set_deterministic(True)
    injected = 0
    for it in range(16):
        t = it * p.dt
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        assert out.np[0] == oo.np[0], (it, out.np[0], oo.np[0])
        assert out.injected[0] == oo.injected[0] and out.removed[0] == oo.removed[0]
        injected += oo.injected[0]
    assert injected > 0
    a, b = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), "particles differ"
    assert np.array_equal(dev.get_currents(), ora.get_currents()), "currents differ"
    assert np.array_equal(dev.get_fields(), ora.get_fields()), "fields differ"


@pytest.mark.parametrize("ndim", [2, 3])
def test_comoving_step_atomic_close(ndim):
    p, dev, ora = _pair(ndim)
    out = dev.lp_run(0.0, 0, initial_time=True)
    rc, oo = ora.lp_run(0.0, 0, initial_time=True)
    assert rc == 0 and out.error_bits == 0 and out.np[0] == oo.np[0]
    a, b = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert _relmax(dev.get_currents(), ora.get_currents()) <= 1e-12
    assert _relmax(dev.get_fields(), ora.get_fields()) <= 1e-12


def test_comoving_needs_fp64():
    p = small_case(2, precision=AGPU_FP32_SPLIT)
    p.w_speed = -VB
    with pytest.raises(AgpuError):
        PicDevice(p)


@pytest.mark.parametrize("ndim", [2, 3])
def test_comoving_env_run_deterministic_bitexact(ndim):
    p, g, ep = env_case(ndim, cap=200000, w_sh=4)
    p.w_speed = -VB
    assert p.precision == AGPU_FP64
    dev = PicDevice(p)
    ora = Oracle(p)
    dev.env_enable(ep)
    ora.env_enable(ep)
    env0 = numpy_init(p, pulse(p, a0=1.5, xc_frac=0.6, wx_frac=0.1, wy_frac=0.3))
    dev.set_envelope(env0)
    ora.set_envelope(env0)
    ebf = 0.02 * laser_fields(p)
    dev.set_fields(ebf)
    ora.set_fields(ebf)
    src = plasma_source(p, x_start_frac=0.7)
    dev.set_plasma_source(src)
    ora.set_plasma_source(src)
    dev.load_plasma(0)
    ora.load_plasma(0)
    dev.set_deterministic(True)
    injected = 0
    for it in range(1, 17):
        t = it * p.dt
        out = dev.env_run(t, it)
        rc, oo = ora.env_run(t, it)
        assert rc == 0 and out.error_bits == 0
        assert out.np[0] == oo.np[0], (it, out.np[0], oo.np[0])
        injected += oo.injected[0]
    assert injected > 0
    a, b = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), "particles differ"
    assert np.array_equal(dev.get_envelope(), ora.get_envelope()), "env differs"
    assert np.array_equal(dev.get_env_source(), ora.get_env_source()), "source scratch differs"
    assert np.array_equal(dev.get_fields(), ora.get_fields()), "fields differ"
