"""Discrete continuity of the device's currents, both precision forms: after
a few laser-driven steps, one more step's currents (agpu_get_currents)
satisfy rho1 - rho0 + c div J_raw = 0 with rho from the particle records
before and after the step (qden shapes, computed on the host in FP64).

Bounds, relative to max |rho|:
* FP64 form: 1e-13 (round-off of the FP64 sums; the atomic deposit only
  reorders them);
* FP32 split form: 1e-6 (FP32 round-off of the shapes and of the
  contributions; the tile sums are exact integers of 2^-30 of the tile's
  scale or finer)."""
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.sim import PicDevice
from tests.test_conservation import conservation_case, residual_after

pytestmark = pytest.mark.gpu

BOUND = {AGPU_FP64: 1e-13, AGPU_FP32_SPLIT: 1e-6}


@pytest.mark.parametrize("precision", [AGPU_FP64, AGPU_FP32_SPLIT])
@pytest.mark.parametrize("ndim,dims", [(3, (64, 32, 32)), (2, (256, 128, 1))])
def test_device_step_conserves_charge(precision, ndim, dims):
    p, src, ebf = conservation_case(ndim, precision, *dims)
    dev = PicDevice(p)
    dev.set_fields(ebf)
    dev.set_plasma_source(src)
    dev.load_plasma(0)
    res, rho, divj = residual_after(dev, p, 5)
    dev.close()
    print(f"ndim {ndim} precision {precision}: residual {res:.3e} = {res / rho:.3e} of max|rho|; "
          f"max|c div J| {divj:.3e}")
    assert divj > 1e-4 * rho
    assert res <= BOUND[precision] * rho, (res / rho, divj / rho)
