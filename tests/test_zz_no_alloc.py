"""The allocation-free field diagnostics entry point.

Hosts that cannot call cudaMalloc (one running inside a CUDA stream capture,
one whose device memory comes from its own pool) get
agpu_field_diag_noalloc: the caller passes the field array already on the
device and a device output of 7 doubles; the entry point's scratch is a
file-scope device array.  This test calls it through the C-ABI twice in a
row -- a 3D grid, then a smaller 2D grid, so a stale partial sum left by the
first call would show in the second -- and checks each result against the
handle-based agpu_diag on the same fields: energies within 1e-12 relative,
max |E| exactly.  It lives in its own file so that it is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from aladyn_b200 import abi
from aladyn_b200.abi import AGPU_E_CAPACITY, AGPU_OK
from aladyn_b200.sim import PicDevice
from tests.helpers import laser_fields, small_case

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, ebf, p):
    d_ebf = torch.from_numpy(np.ascontiguousarray(ebf.ravel(order="F"))).to("cuda")
    d_out = torch.full((7,), -1.0, dtype=torch.float64, device="cuda")
    rc = lib.agpu_field_diag_noalloc(C.c_void_p(d_ebf.data_ptr()), p.ndim, p.nx, p.ny, p.nz, p.dx, p.dy, p.dz,
                                     C.c_void_p(d_out.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == AGPU_OK, rc
    return d_out.cpu().numpy()


def test_field_diag_noalloc_matches_agpu_diag_twice():
    torch = pytest.importorskip("torch")
    lib = abi.load_library()
    for ndim, dims in ((3, (48, 24, 20)), (2, (40, 24, 1))):
        p = small_case(ndim, nx=dims[0], ny=dims[1], nz=dims[2], cap=1000)
        ebf = laser_fields(p)
        dev = PicDevice(p)
        dev.set_fields(ebf)
        ref = dev.diag()
        dev.close()
        out = _noalloc(lib, torch, ebf, p)
        for c in range(p.nfield):
            r = ref.field_energy[c]
            assert abs(out[c] - r) <= 1e-12 * max(abs(r), 1e-300), (ndim, c, out[c], r)
        for c in range(p.nfield, 6):
            assert out[c] == 0.0
        assert out[6] == ref.max_abs_e


def test_field_diag_noalloc_rejects_oversize_grid():
    lib = abi.load_library()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.agpu_field_diag_noalloc(dummy, 3, 1024, 1024, 512, 1.0, 1.0, 1.0, dummy, None)
    assert rc == AGPU_E_CAPACITY
