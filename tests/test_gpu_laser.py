"""The device laser set-up (agpu_init_lp_fields, agpu_init_laser) against the
oracle's restatement of init_lp_inc0_fields (src/fields/init_grid_fields.f90:
406-578, 992-1386) and the host's: FP64 form to 1e-13 of the largest field
(the same FP64 formula; the device's and the host's math libraries may
differ in the last bit), FP32 split form to FP32 rounding (the FP64 pulse
stored in FP32)."""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.config import laser
from aladyn_b200.initial import laser_fields
from aladyn_b200.sim import PicDevice
from oracle.oracle import Oracle
from tests.helpers import LAM0, small_case
from tests.test_laser import _pulse

pytestmark = pytest.mark.gpu

TOL = {AGPU_FP64: 1e-13, AGPU_FP32_SPLIT: 1e-7}


@pytest.mark.parametrize("precision", [AGPU_FP64, AGPU_FP32_SPLIT])
@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("g_prof", [True, False])
def test_device_laser_matches_oracle(precision, ndim, g_prof):
    p = small_case(ndim, precision=precision, nx=96, ny=48, nz=32, cap=16)
    a = _pulse(p, g_prof)
    dev = PicDevice(p)
    dev.init_lp_fields(a)
    fd = dev.get_fields()
    dev.close()
    o = Oracle(small_case(ndim, nx=96, ny=48, nz=32, cap=16))
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    o.init_lp_fields(a)
    fo = o.get_fields()
    assert np.abs(fd - fo).max() <= TOL[precision] * np.abs(fo).max()


def test_init_laser_equals_host_pulse():
    """agpu_init_laser (the namelist form) sets the same fields as the host's
    aladyn_b200.initial.laser_fields, which the CPU baseline runs start from."""
    p = small_case(3, nx=128, ny=48, nz=48, cap=16)
    lx = p.nx * p.dx
    las = laser(3.0, LAM0, 6 * LAM0 / 4, 10 * LAM0 / 4, xc=0.6 * lx, xf=0.7 * lx)
    dev = PicDevice(p)
    dev.init_laser(las)
    fd = dev.get_fields()
    dev.close()
    fh = laser_fields(p, las)
    assert np.abs(fd - fh).max() <= 1e-13 * np.abs(fh).max()
