"""Host logic of the y and y x z decompositions (aladyn_b200/domain.py) on
CPU: the block layout, and the row, plane and particle exchanges of the
block hook driven through a stand-in for the library that keeps each
block's arrays in numpy (the same pack/unpack/emigrant/immigrant contract
as agpu_halo_*), with the thread exchanger and with torch.distributed over
gloo (3 slabs; 2 x 2 blocks, where corner values and corner-crossing
particles must reach the diagonal block).

What the exchanges must give (the reference's fill_ebfield_yzxbdsdata,
fill_curr_yzxbdsdata and part_prl_exchange): after FIELDS every slab's 2
ghost rows on a shared side hold its neighbour's edge rows (all x and z
nodes); after E (B) 2 (1) rows above and 1 (2) below; after CURRENTS every
slab's rows hold the sum of all contributions that fall on them, the sent
ghost rows are zero; after PARTICLES each slab has received the records its
neighbours saw leave towards it."""
import ctypes as C
import os

import numpy as np
import pytest

from aladyn_b200.abi import (AGPU_E_CAPACITY, AGPU_HALO_B, AGPU_HALO_CURRENTS, AGPU_HALO_E, AGPU_HALO_FIELDS,
                             AGPU_HALO_PARTICLES)
from aladyn_b200.config import Grid, make_params
from aladyn_b200.domain import DistExchanger, Slab, SlabLayout, ThreadExchanger, run_threads


def _params(ndim, ny=18, nx=10, nz=6, cap=1000):
    g = Grid(ndim, nx, ny, nz if ndim == 3 else 1, k0=25.0, yx_rat=2.0, zx_rat=2.0, cfl=0.8)
    return make_params(g, capacity=(cap, 0, 0, 0))


def _view(ptr, n):
    return np.ctypeslib.as_array((C.c_double * n).from_address(ptr))


class FakeLib:
    """The agpu_halo_* contract on numpy arrays."""

    def __init__(self):
        self.devs = {}

    def agpu_set_subdomain(self, h, lo, hi, fn, user):
        return 0

    def agpu_set_subdomain_yz(self, h, shared, fn, user):
        self.devs[h].shared = tuple(shared[i] for i in range(4))
        return 0

    def agpu_halo_size_z(self, h, ncomp, nplanes, n):
        d = self.devs[h]
        n._obj.value = ncomp * nplanes * d.n1p * d.n2p
        return 0

    def _block_z(self, d, what, ic1, ic2, k1, n):
        f = d.ebf if what == 0 else d.jc
        return f, (slice(None), slice(None), slice(k1 - 1, k1 - 1 + n), slice(ic1 - 1, ic2))

    def agpu_halo_pack_z(self, h, what, ic1, ic2, k1, n, ptr):
        d = self.devs[h]
        f, sl = self._block_z(d, what, ic1, ic2, k1, n)
        blk = np.transpose(f[sl], (3, 2, 1, 0))  # [component][plane][y][x]
        _view(ptr.value, blk.size)[:] = blk.ravel()
        return 0

    def agpu_halo_unpack_z(self, h, what, ic1, ic2, k1, n, ptr, mode):
        d = self.devs[h]
        f, sl = self._block_z(d, what, ic1, ic2, k1, n)
        shape = f[sl].shape
        if mode == 2:
            f[sl] = 0.0
            return 0
        blk = _view(ptr.value, int(np.prod(shape))).reshape(shape[::-1]).transpose(3, 2, 1, 0)
        f[sl] = blk if mode == 0 else f[sl] + blk
        return 0

    def agpu_halo_size(self, h, ncomp, nrows, n):
        d = self.devs[h]
        n._obj.value = ncomp * nrows * d.n1p * d.n3p
        return 0

    def _block(self, d, what, ic1, ic2, j1, nrows):
        f = d.ebf if what == 0 else d.jc
        return f, (slice(None), slice(j1 - 1, j1 - 1 + nrows), slice(None), slice(ic1 - 1, ic2))

    def agpu_halo_pack(self, h, what, ic1, ic2, j1, nrows, ptr):
        d = self.devs[h]
        f, sl = self._block(d, what, ic1, ic2, j1, nrows)
        blk = np.transpose(f[sl], (3, 2, 1, 0))  # [component][z][row][x]
        _view(ptr.value, blk.size)[:] = blk.ravel()
        return 0

    def agpu_halo_unpack(self, h, what, ic1, ic2, j1, nrows, ptr, mode):
        d = self.devs[h]
        f, sl = self._block(d, what, ic1, ic2, j1, nrows)
        shape = f[sl].shape
        if mode == 2:
            f[sl] = 0.0
            return 0
        blk = _view(ptr.value, int(np.prod(shape))).reshape(shape[::-1]).transpose(3, 2, 1, 0)
        if mode == 0:
            f[sl] = blk
        else:
            f[sl] = f[sl] + blk
        return 0

    def agpu_halo_emigrants(self, h, ic, side, ptr, ld, n):
        d = self.devs[h]
        y = d.part[:, 1]
        if side < 2:
            m = (y <= d.p.gymin) if side == 0 else (y > d.p.gymax)
            if d.p.ndim == 3:
                z = d.part[:, 2]
                zlo, zhi = d.shared[2:] if hasattr(d, "shared") else (0, 0)
                m &= ((z > d.p.gzmin) & (z <= d.p.gzmax)) | ((z <= d.p.gzmin) & bool(zlo)) | \
                    ((z > d.p.gzmax) & bool(zhi))
        else:
            z = d.part[:, 2]
            m = (y > d.p.gymin) & (y <= d.p.gymax) & ((z <= d.p.gzmin) if side == 2 else (z > d.p.gzmax))
        sel = d.part[m]
        n._obj.value = sel.shape[0]
        if sel.shape[0] > ld:
            return AGPU_E_CAPACITY
        out = _view(ptr.value, ld * d.ndv).reshape(d.ndv, ld)
        out[:, :sel.shape[0]] = sel.T
        return 0

    def agpu_halo_immigrants(self, h, ic, ptr, ld, n):
        d = self.devs[h]
        rec = _view(ptr.value, ld * d.ndv).reshape(d.ndv, ld)[:, :n].T
        # the step's compaction drops what left; here the stand-in keeps the
        # records inside the slab, so that forwarded ones do not count twice
        d.part = np.concatenate([d.part, rec])
        return 0


class FakeDev:
    def __init__(self, lib, key, p):
        self.lib = lib
        self.h = key
        self.p = p
        self.n1p, self.n2p = p.nx + 5, p.ny + 5
        self.n3p = p.nz + 5 if p.ndim == 3 else 1
        self.ndv = 7 if p.ndim == 3 else 5
        lib.devs[key] = self

    def stream(self):
        return 0

    def synchronize(self):
        pass


def _global_fields(p, nf, seed=1):
    rng = np.random.default_rng(seed)
    n3p = p.nz + 5 if p.ndim == 3 else 1
    return np.asfortranarray(rng.integers(-50, 50, (p.nx + 5, p.ny + 5, n3p, nf)).astype(np.float64))


def _slabs(p, nslabs, exchanger_for, lib=None):
    lay = SlabLayout(p, nslabs)
    lib = lib or FakeLib()
    slabs = []
    for r in range(nslabs):
        dev = FakeDev(lib, 100 + r, lay.params(r))
        slabs.append(Slab(lay, r, dev, exchanger_for(r), emigrant_capacity=1))
    return lay, slabs


def _local(lay, r, a):
    return np.asfortranarray(a[:, lay.j0[r]:lay.j0[r] + lay.rows[r] + 5].copy())


@pytest.mark.parametrize("ndim", [2, 3])
def test_layout(ndim):
    p = _params(ndim, ny=20)
    lay = SlabLayout(p, 3)
    assert sum(lay.rows) == p.ny and lay.rows == [7, 7, 6]
    ps = [lay.params(r) for r in range(3)]
    assert ps[0].gymin == p.gymin and ps[0].ymn == p.ymn and ps[-1].gymax == p.gymax
    for a, b in zip(ps, ps[1:]):
        assert a.gymax == b.gymin == b.ymn
    for r, q in enumerate(ps):
        assert q.ny == lay.rows[r] and q.nx == p.nx and q.gxmax == p.gxmax
        assert abs(q.gymax - q.gymin - q.ny * p.dy) < 1e-12
    g = _global_fields(p, 3)
    assert np.array_equal(lay.assemble([_local(lay, r, g) for r in range(3)]), g)
    with pytest.raises(ValueError):
        SlabLayout(p, 7)


def _run_point(slabs, point, ic=-1):
    run_threads(slabs, lambda s: _check(s._hook(None, s.dev.h, point, ic)))


def _check(rc):
    assert rc == 0


@pytest.mark.parametrize("ndim", [2, 3])
def test_thread_exchange_fields_e_b(ndim):
    p = _params(ndim)
    nf, nc = (3, 2) if ndim == 2 else (6, 3)
    ex = ThreadExchanger(3)
    lay, slabs = _slabs(p, 3, lambda r: ex)
    g = _global_fields(p, nf)
    for point, down, up, comps in ((AGPU_HALO_FIELDS, 2, 2, range(nf)), (AGPU_HALO_E, 2, 1, range(nc)),
                                   (AGPU_HALO_B, 1, 2, range(nc, nf))):
        for r, s in enumerate(slabs):
            loc = _local(lay, r, g)
            # garbage in the ghost rows of shared sides
            if r > 0:
                loc[:, 0:2] = -999.0
            if r < 2:
                loc[:, -3:] = -999.0
            s.dev.ebf = loc
        _run_point(slabs, point)
        for r, s in enumerate(slabs):
            want = _local(lay, r, g)
            got = s.dev.ebf
            jy1, jy2 = 2, lay.rows[r] + 1           # 0-based
            assert np.array_equal(got[:, jy1:jy2 + 1], want[:, jy1:jy2 + 1])
            for c in range(nf):
                moved = c in comps
                if r > 0:
                    for q in range(1, 3):
                        row = got[:, jy1 - q, :, c]
                        if moved and q <= up:
                            assert np.array_equal(row, want[:, jy1 - q, :, c]), (point, r, c, q)
                        else:
                            assert (row == -999.0).all()
                if r < 2:
                    for q in range(1, 4):
                        row = got[:, jy2 + q, :, c]
                        if moved and q <= down:
                            assert np.array_equal(row, want[:, jy2 + q, :, c]), (point, r, c, q)
                        else:
                            assert (row == -999.0).all()


@pytest.mark.parametrize("ndim", [2, 3])
def test_thread_exchange_currents(ndim):
    p = _params(ndim)
    nc = 2 if ndim == 2 else 3
    ex = ThreadExchanger(3)
    lay, slabs = _slabs(p, 3, lambda r: ex)
    rng = np.random.default_rng(4)
    n3p = p.nz + 5 if ndim == 3 else 1
    total = np.zeros((p.nx + 5, p.ny + 5, n3p, nc), order="F")
    for r, s in enumerate(slabs):
        loc = np.asfortranarray(rng.integers(-20, 20, (p.nx + 5, lay.rows[r] + 5, n3p, nc)).astype(np.float64))
        s.dev.jc = loc.copy(order="F")
        total[:, lay.j0[r]:lay.j0[r] + lay.rows[r] + 5] += loc
    _run_point(slabs, AGPU_HALO_CURRENTS)
    for r, s in enumerate(slabs):
        jy1, jy2 = 2, lay.rows[r] + 1
        got = s.dev.jc
        want = total[:, lay.j0[r]:lay.j0[r] + lay.rows[r] + 5]
        assert np.array_equal(got[:, jy1:jy2 + 1], want[:, jy1:jy2 + 1])
        if r > 0:
            assert not got[:, 0:2].any()
        if r < 2:
            assert not got[:, jy2 + 1:].any()


def _records(p, lay, r, rng, n=30):
    q = lay.params(r)
    ndv = 7 if p.ndim == 3 else 5
    rec = np.zeros((n, ndv))
    rec[:, 0] = rng.uniform(p.gxmin, p.gxmax, n)
    rec[:, 1] = rng.uniform(q.gymin - 0.5 * p.dy, q.gymax + 0.5 * p.dy, n)
    rec[:, -1] = np.arange(n) + 1000 * r
    return rec


def test_thread_exchange_particles():
    p = _params(2)
    ex = ThreadExchanger(3)
    lay, slabs = _slabs(p, 3, lambda r: ex)
    rng = np.random.default_rng(7)
    start = []
    for r, s in enumerate(slabs):
        s.dev.part = _records(p, lay, r, rng)
        start.append(s.dev.part.copy())
    _run_point(slabs, AGPU_HALO_PARTICLES, 0)
    for r, s in enumerate(slabs):
        q = lay.params(r)
        arrived = s.dev.part[start[r].shape[0]:]
        want = []
        if r > 0:   # from below: the low neighbour's records above its gymax
            lo = start[r - 1]
            want.append(lo[lo[:, 1] > lay.params(r - 1).gymax])
        if r < 2:
            hi = start[r + 1]
            want.append(hi[hi[:, 1] <= lay.params(r + 1).gymin])
        want = np.concatenate(want) if want else np.zeros((0, 5))
        key = lambda a: a[np.argsort(a[:, -1])]
        assert np.array_equal(key(arrived), key(want))
        assert ((arrived[:, 1] > q.gymin) & (arrived[:, 1] <= q.gymax)).all()
        assert s.migrated == arrived.shape[0]
    # more records than the first emigrant buffer held: the buffer grew
    assert max(s.ecap for s in slabs) > 1


def _gloo_worker(rank, world, port, ndim, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _params(ndim)
        nf = 3 if ndim == 2 else 6
        nc = nf // 2
        lay = SlabLayout(p, world)
        lib = FakeLib()
        dev = FakeDev(lib, 100 + rank, lay.params(rank))
        slab = Slab(lay, rank, dev, DistExchanger(), emigrant_capacity=4)
        g = _global_fields(p, nf)
        loc = _local(lay, rank, g)
        if rank > 0:
            loc[:, 0:2] = -999.0
        if rank < world - 1:
            loc[:, -3:] = -999.0
        dev.ebf = loc
        assert slab._hook(None, dev.h, AGPU_HALO_FIELDS, -1) == 0, slab.error
        want = _local(lay, rank, g)
        ok_fields = np.array_equal(dev.ebf[:, :lay.rows[rank] + 4], want[:, :lay.rows[rank] + 4])
        # currents: integer-valued, the sums are exact
        rng = np.random.default_rng(11)
        n3p = p.nz + 5 if ndim == 3 else 1
        total = np.zeros((p.nx + 5, p.ny + 5, n3p, nc), order="F")
        mine = None
        for r in range(world):
            a = np.asfortranarray(rng.integers(-9, 9, (p.nx + 5, lay.rows[r] + 5, n3p, nc)).astype(np.float64))
            total[:, lay.j0[r]:lay.j0[r] + lay.rows[r] + 5] += a
            if r == rank:
                mine = a
        dev.jc = mine.copy(order="F")
        assert slab._hook(None, dev.h, AGPU_HALO_CURRENTS, -1) == 0, slab.error
        jy2 = lay.rows[rank] + 1
        ok_curr = np.array_equal(dev.jc[:, 2:jy2 + 1], total[:, lay.j0[rank] + 2:lay.j0[rank] + jy2 + 1])
        # particles
        rng = np.random.default_rng(5)
        recs = [_records(p, lay, r, rng) for r in range(world)]
        dev.part = recs[rank].copy()
        assert slab._hook(None, dev.h, AGPU_HALO_PARTICLES, 0) == 0, slab.error
        n_in = 0
        if rank > 0:
            n_in += int((recs[rank - 1][:, 1] > lay.params(rank - 1).gymax).sum())
        if rank < world - 1:
            n_in += int((recs[rank + 1][:, 1] <= lay.params(rank + 1).gymin).sum())
        ok_part = dev.part.shape[0] == recs[rank].shape[0] + n_in and slab.migrated == n_in
        out.put((rank, ok_fields, ok_curr, ok_part))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ndim", [2, 3])
def test_dist_exchanger_gloo(ndim):
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 3
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, ndim, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, ok_f, ok_c, ok_p in sorted(res):
        assert ok_f and ok_c and ok_p, (rank, ok_f, ok_c, ok_p)


# ---- y and z split (2 x 2 blocks, 3D) ------------------------------------------
def _blocks(p, ny_s, nz_s, ex):
    lay = SlabLayout(p, ny_s, nz_s)
    lib = FakeLib()
    blocks = []
    for r in range(lay.n):
        dev = FakeDev(lib, 200 + r, lay.params(r))
        blocks.append(Slab(lay, r, dev, ex, emigrant_capacity=1))
    return lay, blocks


def test_yz_layout():
    p = _params(3, ny=18, nz=14)
    lay = SlabLayout(p, 2, 2)
    assert lay.n == 4 and lay.rows == [9, 9] and lay.planes == [7, 7]
    q = [lay.params(r) for r in range(4)]
    assert q[0].gzmin == p.gzmin and q[2].gzmax == p.gzmax and q[0].gzmax == q[2].gzmin == q[2].zmn
    assert q[0].gymax == q[1].gymin and q[0].nz == 7 and q[3].ny == 9
    assert lay.shared(0) == (False, True, False, True) and lay.shared(3) == (True, False, True, False)
    assert lay.neighbours(0) == {1: 1, 3: 2} and lay.neighbours(3) == {0: 2, 2: 1}
    g = _global_fields(p, 6)
    assert np.array_equal(lay.assemble([lay.local(r, g) for r in range(4)]), g)


def test_yz_exchange_fields_with_corners():
    p = _params(3, ny=18, nz=14)
    ex = ThreadExchanger(4)
    lay, blocks = _blocks(p, 2, 2, ex)
    g = _global_fields(p, 6)
    for r, b in enumerate(blocks):
        loc = lay.local(r, g).copy(order="F")
        lo, hi, zlo, zhi = lay.shared(r)
        if lo:
            loc[:, 0:2] = -999.0
        if hi:
            loc[:, -3:] = -999.0
        if zlo:
            loc[:, :, 0:2] = -999.0
        if zhi:
            loc[:, :, -3:] = -999.0
        b.dev.ebf = loc
    _run_point(blocks, AGPU_HALO_FIELDS)
    for r, b in enumerate(blocks):
        want = lay.local(r, g)
        got = b.dev.ebf
        ry, rz = lay.coords(r)
        nr, nk = lay.rows[ry], lay.planes[rz]
        # every node within 2 layers of the interior, corners included
        sl = (slice(None), slice(0, nr + 4), slice(0, nk + 4))
        assert np.array_equal(got[sl], want[sl]), r


def test_yz_exchange_currents_with_corners():
    p = _params(3, ny=18, nz=14)
    ex = ThreadExchanger(4)
    lay, blocks = _blocks(p, 2, 2, ex)
    rng = np.random.default_rng(9)
    total = np.zeros((p.nx + 5, p.ny + 5, p.nz + 5, 3), order="F")
    for r, b in enumerate(blocks):
        ry, rz = lay.coords(r)
        shape = (p.nx + 5, lay.rows[ry] + 5, lay.planes[rz] + 5, 3)
        loc = np.asfortranarray(rng.integers(-20, 20, shape).astype(np.float64))
        b.dev.jc = loc.copy(order="F")
        total[:, lay.j0[ry]:lay.j0[ry] + lay.rows[ry] + 5, lay.k0[rz]:lay.k0[rz] + lay.planes[rz] + 5] += loc
    _run_point(blocks, AGPU_HALO_CURRENTS)
    for r, b in enumerate(blocks):
        ry, rz = lay.coords(r)
        nr, nk = lay.rows[ry], lay.planes[rz]
        want = total[:, lay.j0[ry]:lay.j0[ry] + nr + 5, lay.k0[rz]:lay.k0[rz] + nk + 5]
        got = b.dev.jc
        assert np.array_equal(got[:, 2:nr + 2, 2:nk + 2], want[:, 2:nr + 2, 2:nk + 2]), r


def test_yz_exchange_particles_reach_the_diagonal_block():
    p = _params(3, ny=18, nz=14)
    ex = ThreadExchanger(4)
    lay, blocks = _blocks(p, 2, 2, ex)
    rng = np.random.default_rng(21)
    start = []
    for r, b in enumerate(blocks):
        q = lay.params(r)
        n = 60
        rec = np.zeros((n, 7))
        rec[:, 0] = rng.uniform(p.gxmin, p.gxmax, n)
        rec[:, 1] = rng.uniform(q.gymin - 0.5 * p.dy, q.gymax + 0.5 * p.dy, n)
        rec[:, 2] = rng.uniform(q.gzmin - 0.5 * p.dz, q.gzmax + 0.5 * p.dz, n)
        rec[:, -1] = np.arange(n) + 1000 * r
        b.dev.part = rec
        start.append(rec.copy())
    _run_point(blocks, AGPU_HALO_PARTICLES, 0)
    allrec = np.concatenate(start)
    for r, b in enumerate(blocks):
        q = lay.params(r)
        inside = (b.dev.part[:, 1] > q.gymin) & (b.dev.part[:, 1] <= q.gymax) & \
            (b.dev.part[:, 2] > q.gzmin) & (b.dev.part[:, 2] <= q.gzmax)
        got = np.sort(b.dev.part[inside, -1])
        # every record that lies in this block after the exchange, whichever block it started in
        m = (allrec[:, 1] > q.gymin) & (allrec[:, 1] <= q.gymax) & (allrec[:, 2] > q.gzmin) & (allrec[:, 2] <= q.gzmax)
        assert np.array_equal(got, np.sort(allrec[m, -1])), r
    # some records crossed a corner (both a y and a z side)
    diag = 0
    for r in range(4):
        q = lay.params(r)
        y, z = start[r][:, 1], start[r][:, 2]
        diag += int((((y <= q.gymin) | (y > q.gymax)) & ((z <= q.gzmin) | (z > q.gzmax))).sum())
    assert diag > 0


def _gloo_yz_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _params(3, ny=18, nz=14)
        lay = SlabLayout(p, 2, 2)
        lib = FakeLib()
        dev = FakeDev(lib, 300 + rank, lay.params(rank))
        blk = Slab(lay, rank, dev, DistExchanger(), emigrant_capacity=2)
        g = _global_fields(p, 6)
        loc = lay.local(rank, g).copy(order="F")
        lo, hi, zlo, zhi = lay.shared(rank)
        if lo:
            loc[:, 0:2] = -999.0
        if hi:
            loc[:, -3:] = -999.0
        if zlo:
            loc[:, :, 0:2] = -999.0
        if zhi:
            loc[:, :, -3:] = -999.0
        dev.ebf = loc
        assert blk._hook(None, dev.h, AGPU_HALO_FIELDS, -1) == 0, blk.error
        ry, rz = lay.coords(rank)
        nr, nk = lay.rows[ry], lay.planes[rz]
        sl = (slice(None), slice(0, nr + 4), slice(0, nk + 4))
        ok_f = np.array_equal(dev.ebf[sl], lay.local(rank, g)[sl])
        # particles: every record that ends inside a block is there once
        rng = np.random.default_rng(8)
        recs = []
        for r in range(world):
            q = lay.params(r)
            a = np.zeros((40, 7))
            a[:, 0] = rng.uniform(p.gxmin, p.gxmax, 40)
            a[:, 1] = rng.uniform(q.gymin - 0.5 * p.dy, q.gymax + 0.5 * p.dy, 40)
            a[:, 2] = rng.uniform(q.gzmin - 0.5 * p.dz, q.gzmax + 0.5 * p.dz, 40)
            a[:, -1] = np.arange(40) + 1000 * r
            recs.append(a)
        dev.part = recs[rank].copy()
        assert blk._hook(None, dev.h, AGPU_HALO_PARTICLES, 0) == 0, blk.error
        q = lay.params(rank)
        inside = lambda a: (a[:, 1] > q.gymin) & (a[:, 1] <= q.gymax) & (a[:, 2] > q.gzmin) & (a[:, 2] <= q.gzmax)
        allrec = np.concatenate(recs)
        ok_p = np.array_equal(np.sort(dev.part[inside(dev.part), -1]), np.sort(allrec[inside(allrec), -1]))
        out.put((rank, ok_f, ok_p))
    finally:
        dist.destroy_process_group()


def test_dist_exchanger_gloo_yz_blocks():
    """2 x 2 blocks over torch.distributed (gloo, 4 ranks): field halos with
    corners and particles reaching the diagonal block."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_yz_worker, args=(r, 4, port, q)) for r in range(4)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in range(4)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, ok_f, ok_p in sorted(res):
        assert ok_f and ok_p, (rank, ok_f, ok_p)
