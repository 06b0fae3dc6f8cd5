"""The device's envelope cycle (agpu_env_run: env_lpf2_evolve + the moving
window, src/dynamics/env_evolve_in_time.f90:196-391) against the oracle.

Tolerances:
* deterministic mode (serial density and current sums): env, the source
  scratch, fields, currents and particles bit-exact after 22 steps with two
  window shifts, in 2D and 3D, der_ord 2 and 3;
* atomic sums (the density and currents differ by the order of the FP64
  sums, which reaches the envelope through the plasma source; the records
  are kept in tile order): particle count equal, each particle column as a
  sorted set, env and fields to 1e-12 of their largest value after 8 steps;
* the pulse set-up (agpu_init_envelope): 1e-13 of the largest value (the
  device's and the host's math libraries may differ in the last bit).
"""
import numpy as np
import pytest

from aladyn_b200.sim import PicDevice
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source
from tests.test_envelope import env_case, numpy_init, pulse

pytestmark = pytest.mark.gpu


def _pair(ndim, der_ord=2, nx=64, ny=24, nz=16, w_sh=10, iform=0):
    p, g, ep = env_case(ndim, nx=nx, ny=ny, nz=nz, der_ord=der_ord, cap=200000, w_sh=w_sh)
    p.iform = iform
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
    src = plasma_source(p, x_start_frac=0.3)
    dev.set_plasma_source(src)
    ora.set_plasma_source(src)
    dev.load_plasma(0)
    ora.load_plasma(0)
    return p, dev, ora


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("g_prof,plane_wave", [(True, False), (False, False), (True, True)])
def test_init_envelope_matches_oracle(ndim, g_prof, plane_wave):
    p, g, ep = env_case(ndim)
    a = pulse(p, g_prof=g_prof)
    dev = PicDevice(p)
    dev.env_enable(ep)
    dev.init_envelope(a, plane_wave)
    got = dev.get_envelope()
    dev.close()
    o = Oracle(p)
    o.env_enable(ep)
    o.init_envelope(a, plane_wave)
    want = o.get_envelope()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("der_ord", [2, 3])
def test_env_run_deterministic_bitexact(ndim, der_ord):
    p, dev, ora = _pair(ndim, der_ord)
    dev.set_deterministic(True)
    n0 = ora.count(0)
    assert n0 > 1000
    shifts = 0
    for it in range(1, 23):
        t = it * p.dt
        out = dev.env_run(t, it)
        rc, oo = ora.env_run(t, it)
        assert rc == 0 and out.error_bits == 0
        assert out.np[0] == oo.np[0], (it, out.np[0], oo.np[0])
        assert out.nshx == oo.nshx
        shifts += out.nshx > 0
    assert shifts == 2
    assert dev.window_state()[3] == ora.xmn()
    a, b = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), "particles differ"
    assert np.array_equal(dev.get_envelope(), ora.get_envelope()), "env differs"
    assert np.array_equal(dev.get_env_source(), ora.get_env_source()), "source scratch differs"
    assert np.array_equal(dev.get_fields(), ora.get_fields()), "fields differ"
    assert np.array_equal(dev.get_currents(), ora.get_currents()), "currents differ"
    # the plasma has felt the pulse
    assert np.abs(a[:, ndim:2 * ndim]).max() > 1e-3


@pytest.mark.parametrize("ndim", [2, 3])
def test_env_run_iform2_deterministic_bitexact(ndim):
    """The envelope cycle with the iform = 2 deposit (lpf_env_positions keeps
    dt / gamma for it): bit-exact over 12 steps with a window shift."""
    p, dev, ora = _pair(ndim, iform=2)
    dev.set_deterministic(True)
    for it in range(1, 13):
        out = dev.env_run(it * p.dt, it)
        rc, oo = ora.env_run(it * p.dt, it)
        assert rc == 0 and out.error_bits == 0 and out.np[0] == oo.np[0]
    a, b = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert np.array_equal(dev.get_currents(), ora.get_currents())
    assert np.array_equal(dev.get_fields(), ora.get_fields())
    assert np.array_equal(dev.get_envelope(), ora.get_envelope())


@pytest.mark.parametrize("ndim", [2, 3])
def test_env_run_atomic_close(ndim):
    p, dev, ora = _pair(ndim)
    out = dev.env_run(p.dt, 1)
    rc, oo = ora.env_run(p.dt, 1)
    assert rc == 0 and out.error_bits == 0 and out.np[0] == oo.np[0]
    for it in range(2, 9):
        dev.env_run(it * p.dt, it)
        ora.env_run(it * p.dt, it)
    assert _relmax(dev.get_envelope(), ora.get_envelope()) <= 1e-12
    assert _relmax(dev.get_fields(), ora.get_fields()) <= 1e-12
    # the atomic mode keeps its records in tile order: compare each column
    # as a sorted set
    a, b = dev.get_species(0), ora.get_species(0)
    assert a.shape == b.shape
    for c in range(2 * ndim):
        assert _relmax(np.sort(a[:, c]), np.sort(b[:, c])) <= 1e-12, c


def test_env_requires_enable_and_fp64():
    p, g, ep = env_case(2)
    dev = PicDevice(p)
    with pytest.raises(RuntimeError):
        dev.env_run(p.dt, 1)
    dev.close()
    from aladyn_b200.abi import AGPU_FP32_SPLIT
    from tests.helpers import small_case
    q = small_case(2, precision=AGPU_FP32_SPLIT, nx=64, ny=24, cap=1000)
    d32 = PicDevice(q)
    with pytest.raises(RuntimeError):
        d32.env_enable(ep)
    d32.close()
