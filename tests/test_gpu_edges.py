"""Edge cases of the device step, both forms, against the oracle:

* no particles at all through a window shift: no counts, no error bits,
  fields as the oracle's (vacuum update and field shift);
* box-edge removal (reset_all_part_dist, mpi_part_interface.f90:467-523):
  at rest in zero fields a record exactly on the right box edge stays, one
  just beyond it and one exactly on the left edge leave.
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.sim import PicDevice, pack_slot
from oracle.oracle import Oracle
from tests.helpers import laser_fields, small_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("precision,tol", [(AGPU_FP64, 1e-12), (AGPU_FP32_SPLIT, 1e-5)])
def test_empty_species_with_window(ndim, precision, tol):
    p = small_case(ndim, precision=precision, nx=40, ny=20, nz=12, cap=1000)
    dev = PicDevice(p)
    ora = Oracle(small_case(ndim, nx=40, ny=20, nz=12, cap=1000))
    ebf = laser_fields(p)
    dev.set_fields(ebf)
    ora.set_fields(ebf)
    t = 0.0
    for it in range(12):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert out.error_bits == 0 and out.np[0] == 0
        assert out.nshx == oo.nshx
        t += p.dt
    fa, fb = dev.get_fields(), ora.get_fields()
    assert np.abs(fa - fb).max() <= tol * np.abs(fb).max()
    assert dev.count(0) == 0


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("precision", [AGPU_FP64, AGPU_FP32_SPLIT])
def test_box_edge_removal(ndim, precision):
    p = small_case(ndim, precision=precision, nx=40, ny=20, nz=12, cap=1000)
    dev = PicDevice(p)
    dev.set_fields(np.zeros_like(laser_fields(p)))
    yc = 0.5 * (p.gymin + p.gymax)
    zc = 0.5 * (p.gzmin + p.gzmax)
    xs = [p.gxmax, p.gxmax + 1e-9 * p.dx, p.gxmin, 0.5 * (p.gxmin + p.gxmax)]
    rec = np.zeros((len(xs), 2 * ndim + 1))
    rec[:, 0] = xs
    rec[:, 1] = yc
    if ndim == 3:
        rec[:, 2] = zc
    rec[:, -1] = pack_slot(-1, 0, 1.0)
    dev.set_species(0, rec)
    out = dev.lp_run(0.0, 1)  # no window shift on iteration 1
    assert out.error_bits == 0
    kept = dev.get_species(0)
    assert kept.shape[0] == 2
    want = sorted([p.gxmax, xs[3]])
    got = sorted(kept[:, 0].tolist())
    assert np.allclose(got, want, rtol=0, atol=1e-6 * p.dx)


@pytest.mark.parametrize("precision", [AGPU_FP64, AGPU_FP32_SPLIT])
def test_capacity_limits(precision):
    """A species that would outgrow its capacity is refused with
    AGPU_E_CAPACITY (records, plasma load, window injection) before anything
    is written past the arrays; the records already set stay intact."""
    from aladyn_b200.abi import AGPU_E_CAPACITY, AgpuError
    from tests.helpers import plasma_source
    ndim = 3
    p = small_case(ndim, precision=precision, nx=40, ny=20, nz=12, cap=1000)
    dev = PicDevice(p)
    dev.set_fields(laser_fields(p))
    yc = 0.5 * (p.gymin + p.gymax)
    rec = np.zeros((1001, 2 * ndim + 1))
    rec[:, 0] = np.linspace(p.gxmin + p.dx, p.gxmax - p.dx, 1001)
    rec[:, 1] = yc
    rec[:, 2] = 0.5 * (p.gzmin + p.gzmax)
    rec[:, -1] = pack_slot(-1, 0, 1.0)
    with pytest.raises(AgpuError) as e:
        dev.set_species(0, rec)
    assert e.value.code == AGPU_E_CAPACITY
    dev.set_species(0, rec[:1000])
    with pytest.raises(AgpuError) as e:
        dev.window_inject(0, rec[:1])
    assert e.value.code == AGPU_E_CAPACITY
    dev.set_plasma_source(plasma_source(p))
    with pytest.raises(AgpuError) as e:
        dev.load_plasma(0)
    assert e.value.code == AGPU_E_CAPACITY
    back = dev.get_species(0)
    assert back.shape[0] == 1000
    assert np.abs(back[:, 0] - rec[:1000, 0]).max() <= 1e-6 * p.dx
