"""Stretched transverse grids on the device (agpu_set_stretch) against the
oracle: FP64 form, per-particle kernels, a laser and particles spread over
the whole box (uniform middle and both stretched ends in y, and z in 3D).

Tolerance: 1e-12 of the largest value after 10 steps (fields, currents,
particle records) in the deterministic mode.  The particle map uses atan,
whose device and host implementations may differ in the last bit; every
other operation is the oracle's, in its order.  Refusals: the split form,
a plasma lattice source (stretched targets come from the host), the
envelope cycle."""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AgpuError
from aladyn_b200.config import StretchedGrid, env_params
from aladyn_b200.sim import PicDevice, pack_slot
from oracle.oracle import Oracle
from tests.helpers import grid_small, laser_fields, plasma_source, small_case

pytestmark = pytest.mark.gpu


def _records(p, n=20000, seed=3):
    rng = np.random.default_rng(seed)
    nd = 7 if p.ndim == 3 else 5
    rec = np.zeros((n, nd), order="F")
    rec[:, 0] = rng.uniform(p.gxmin + 4 * p.dx, p.gxmax - 4 * p.dx, n)
    span = p.gymax - p.gymin
    rec[:, 1] = rng.uniform(p.gymin + 0.02 * span, p.gymax - 0.02 * span, n)
    if p.ndim == 3:
        zspan = p.gzmax - p.gzmin
        rec[:, 2] = rng.uniform(p.gzmin + 0.02 * zspan, p.gzmax - 0.02 * zspan, n)
    rec[:, p.ndim:2 * p.ndim] = rng.normal(0.0, 0.3, (n, p.ndim))
    rec[:, -1] = pack_slot(-1, 0, 0.5)
    return rec


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ndim,str_flag", [(2, 1), (2, 2), (3, 1)])
def test_stretched_step_matches_oracle(ndim, str_flag):
    p = small_case(ndim, nx=48, ny=48, nz=32, w_sh=0)
    sg = StretchedGrid(p, str_flag)
    dev = PicDevice(p)
    ora = Oracle(p)
    dev.set_stretch(sg)
    ora.set_stretch(sg)
    ebf = laser_fields(p, a0=1.0)
    dev.set_fields(ebf)
    ora.set_fields(ebf)
    rec = _records(p)
    dev.set_species(0, rec)
    ora.set_species(0, rec)
    dev.set_deterministic(True)
    t = 0.0
    for it in range(10):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0 and oo.error_bits == 0
        assert out.np[0] == oo.np[0], (it, out.np[0], oo.np[0])
        t += p.dt
    a, b = dev.get_species(0), ora.get_species(0)
    err_p = np.abs(a - b).max(axis=0) / np.maximum(np.abs(b).max(axis=0), 1e-300)
    err_f = _relmax(dev.get_fields(), ora.get_fields())
    err_j = _relmax(dev.get_currents(), ora.get_currents())
    print(f"ndim {ndim} str_flag {str_flag}: particles {err_p.max():.2e} fields {err_f:.2e} currents {err_j:.2e}")
    assert err_p.max() <= 1e-12 and err_f <= 1e-12 and err_j <= 1e-12
    # the stretched ends carried particles
    ys = (b[:, 1] < sg.y["smin"]) | (b[:, 1] > sg.y["smax"])
    assert ys.sum() > 100


def test_stretch_refusals():
    p = small_case(2, precision=AGPU_FP32_SPLIT)
    sg = StretchedGrid(p, 1)
    dev = PicDevice(p)
    with pytest.raises(AgpuError):
        dev.set_stretch(sg)
    p = small_case(2)
    sg = StretchedGrid(p, 1)
    dev = PicDevice(p)
    dev.set_plasma_source(plasma_source(p))
    with pytest.raises(AgpuError):
        dev.set_stretch(sg)
    dev = PicDevice(p)
    dev.set_stretch(sg)
    with pytest.raises(AgpuError):
        dev.set_plasma_source(plasma_source(p))
    with pytest.raises(AgpuError):
        dev.env_enable(env_params(grid_small(2), 0.8))
