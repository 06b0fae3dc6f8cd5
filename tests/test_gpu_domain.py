"""The y (and y x z) decomposition on the device (agpu_set_subdomain,
agpu_set_subdomain_yz + the slab hook of aladyn_b200/domain.py) against one
box: 2 and 3 slabs, and 2 x 2 blocks in 3D, of one simulation on one GPU,
one host thread per block (the threads meet at barriers between kernels;
no kernel waits on another), FP64 form.

Tolerances: the plasma load is the same particle set bit for bit (each
slab keeps the lattice particles of its rows); after 14 steps with a window
shift the particle counts are equal, and fields, currents and particles
agree with one box to 1e-10 of their largest value: the slabs add the ghost
currents of their neighbours after their own (one box adds them in deposit
order) and gather with local coordinates y - ymn_slab, so the sums differ in
the last bits, which the steps carry along."""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_E_STATE, AGPU_FP32_SPLIT, AgpuError
from aladyn_b200.domain import Slab, SlabLayout, ThreadExchanger, run_threads
from aladyn_b200.sim import PicDevice
from tests.helpers import laser_fields, plasma_source, small_case

pytestmark = pytest.mark.gpu


def _key(rec, scale):
    r = np.round(rec / scale, 8)
    return rec[np.lexsort(r.T[::-1])]


def _setup(ndim, nslabs, nzslabs=1):
    p = small_case(ndim, w_sh=10)
    lay = SlabLayout(p, nslabs, nzslabs)
    ebf = laser_fields(p)
    src = plasma_source(p, x_start_frac=0.3)
    one = PicDevice(p)
    one.set_fields(ebf)
    one.set_plasma_source(src)
    one.load_plasma(0)
    ex = ThreadExchanger(lay.n)
    slabs = []
    for r in range(lay.n):
        dev = PicDevice(lay.params(r))
        dev.set_fields(lay.local(r, ebf))
        dev.set_plasma_source(src)
        slabs.append(Slab(lay, r, dev, ex))
        dev.load_plasma(0)
    return p, lay, one, slabs


def _union(slabs):
    return np.concatenate([s.dev.get_species(0) for s in slabs])


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ndim,nslabs,nzslabs", [(2, 2, 1), (2, 3, 1), (3, 2, 1), (3, 3, 1), (3, 2, 2)])
def test_slabs_match_one_box(ndim, nslabs, nzslabs):
    p, lay, one, slabs = _setup(ndim, nslabs, nzslabs)
    nblocks = lay.n
    a0, b0 = _union(slabs), one.get_species(0)
    assert a0.shape == b0.shape and a0.shape[0] > 1000
    order = lambda a: a[np.lexsort(a.T[::-1])]
    assert np.array_equal(order(a0), order(b0)), "the slabs' plasma load differs from one box"
    shifts = 0
    for it in range(14):
        t = it * p.dt
        o1 = one.lp_run(t, it, initial_time=(it == 0))
        outs = [None] * nblocks

        def step(s):
            outs[s.rank] = s.dev.lp_run(t, it, initial_time=(it == 0))

        run_threads(slabs, step)
        assert o1.error_bits == 0 and all(o.error_bits == 0 for o in outs)
        assert sum(o.np[0] for o in outs) == o1.np[0], it
        assert all(o.nshx == o1.nshx for o in outs)
        shifts += o1.nshx > 0
    assert shifts >= 1
    assert sum(s.migrated for s in slabs) > 0, "no particle crossed a slab boundary"
    for s in slabs:
        assert s.calls[1] == 14 and s.calls[3] == 14 and s.calls[4] == 28 and s.calls[5] == 14
    f_one = one.get_fields()
    f_dd = lay.assemble([s.dev.get_fields() for s in slabs])
    err_f = _relmax(f_dd, f_one)
    j_one = one.get_currents()
    j_dd = lay.assemble([s.dev.get_currents() for s in slabs])
    # the assembled interior (ghost layers at shared sides are zero in the blocks)
    kin = slice(2, p.nz + 2) if ndim == 3 else slice(0, 1)
    err_j = _relmax(j_dd[:, 2:p.ny + 2, kin], j_one[:, 2:p.ny + 2, kin])
    a, b = _union(slabs), one.get_species(0)
    assert a.shape == b.shape
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    ka, kb = _key(a, scale), _key(b, scale)
    err_p = (np.abs(ka - kb) / scale).max()
    print(f"ndim {ndim} blocks {nslabs}x{nzslabs}: fields {err_f:.2e} currents {err_j:.2e} particles {err_p:.2e}")
    assert err_f <= 1e-10 and err_j <= 1e-10 and err_p <= 1e-10


def test_halo_pack_unpack_roundtrip():
    import torch
    p = small_case(3)
    lay = SlabLayout(p, 2)
    ebf = laser_fields(p)
    dev = PicDevice(lay.params(0))
    loc = np.asfortranarray(ebf[:, 0:lay.rows[0] + 5])
    dev.set_fields(loc)
    lib = dev.lib
    import ctypes as C
    n = C.c_int64()
    assert lib.agpu_halo_size(dev.h, 2, 3, C.byref(n)) == 0
    buf = torch.empty(n.value, dtype=torch.float64, device="cuda")
    assert lib.agpu_halo_pack(dev.h, 0, 2, 3, 4, 3, C.c_void_p(buf.data_ptr())) == 0
    dev.synchronize()
    want = np.transpose(loc[:, 3:6, :, 1:3], (3, 2, 1, 0)).ravel()
    assert np.array_equal(buf.cpu().numpy(), want)
    # write the block two rows lower, add it, zero it
    assert lib.agpu_halo_unpack(dev.h, 0, 2, 3, 1, 3, C.c_void_p(buf.data_ptr()), 0) == 0
    got = dev.get_fields()
    assert np.array_equal(got[:, 0:3, :, 1:3], loc[:, 3:6, :, 1:3])
    assert lib.agpu_halo_unpack(dev.h, 0, 2, 3, 1, 3, C.c_void_p(buf.data_ptr()), 1) == 0
    assert np.array_equal(dev.get_fields()[:, 0:3, :, 1:3], 2 * loc[:, 3:6, :, 1:3])
    assert lib.agpu_halo_unpack(dev.h, 0, 2, 3, 1, 3, None, 2) == 0
    assert not dev.get_fields()[:, 0:3, :, 1:3].any()
    # rows past the array and unknown arrays are refused
    assert lib.agpu_halo_pack(dev.h, 0, 1, 1, lay.rows[0] + 5, 2, C.c_void_p(buf.data_ptr())) != 0
    assert lib.agpu_halo_pack(dev.h, 2, 1, 1, 1, 1, C.c_void_p(buf.data_ptr())) != 0


def test_subdomain_refusals():
    from aladyn_b200.abi import HALO_FN
    fn = HALO_FN(lambda u, h, point, ic: 0)
    dev32 = PicDevice(small_case(2, precision=AGPU_FP32_SPLIT))
    assert dev32.lib.agpu_set_subdomain(dev32.h, 1, 0, fn, None) != 0
    dev = PicDevice(small_case(2))
    assert dev.lib.agpu_set_subdomain(dev.h, 1, 0, fn, None) == 0
    assert dev.lib.agpu_set_step_graphs(dev.h, 1) == AGPU_E_STATE
    assert dev.lib.agpu_set_fused_yee(dev.h, 1) == AGPU_E_STATE
    from aladyn_b200.config import env_params
    from tests.helpers import grid_small
    with pytest.raises(AgpuError):
        dev.env_enable(env_params(grid_small(2), 0.8))
