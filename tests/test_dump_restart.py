"""Dump / restart in the reference's dumpRestart formats (dump_data /
restart, src/start/pic_dump.f90), CPU checks with the oracle as the state
holder (the device holder, PicDevice, exposes the same calls):

* Fortran unformatted sequential records: markers, round trip, corruption
  detected;
* a dump written and read back gives the same arrays and scalars, with the
  reference's record layout in Comm-data.bin;
* a run dumped after a window shift and restarted in a fresh state holder
  continues bit for bit like the uninterrupted run, through the next window
  shift and injection;
* a dump without the window counter (rdata(10) = 0, as the reference
  writes it) restarts the window counters from zero, as the reference does.
"""
import math
import os

import numpy as np
import pytest

from aladyn_b200 import dump
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case


def test_fortran_records_round_trip(tmp_path):
    path = str(tmp_path / "r.bin")
    recs = [np.arange(10, dtype=np.float64), np.arange(7, dtype=np.int32), np.array([1.5, -2.0])]
    dump.write_records(path, recs)
    raw = open(path, "rb").read()
    assert len(raw) == sum(r.nbytes + 8 for r in recs)
    assert np.frombuffer(raw[:4], dtype=np.int32)[0] == 80
    back = dump.read_records(path)
    assert [np.frombuffer(b, dtype=r.dtype).tolist() for b, r in zip(back, recs)] == [r.tolist() for r in recs]
    bad = bytearray(raw)
    bad[84] ^= 0xFF  # trailing marker of the first record
    open(path, "wb").write(bytes(bad))
    with pytest.raises(ValueError):
        dump.read_records(path)


def _run(p, src, steps, t=0.0, it0=0, holder=None):
    o = holder
    for it in range(it0, it0 + steps):
        rc, out = o.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        t += p.dt
    return t


def _fresh(ndim):
    p = small_case(ndim, nx=40, ny=20, nz=12, cap=120_000)
    src = plasma_source(p)
    src.x_end = p.xmax + 40 * p.dx  # a target 40 cells beyond the box: a short xpt table
    o = Oracle(p)
    o.set_fields(laser_fields(p))
    o.set_plasma_source(src)
    o.load_plasma(0)
    return p, src, o


@pytest.mark.parametrize("ndim", [2, 3])
def test_dump_files_round_trip(ndim, tmp_path):
    p, src, o = _fresh(ndim)
    t = _run(p, src, 12, holder=o)
    st = dump.capture(o, p, 12, t, [src])
    xmax = p.xmax + st.x0
    dump.write_dump(str(tmp_path), st, xmax)
    recs = dump.read_records(str(tmp_path / dump.COMM))
    nptx_max = st.xpt.shape[0]
    assert [len(r) for r in recs[:4]] == [80, 40, 4, 4]
    assert len(recs) == 4 + nptx_max + 3 and all(len(r) == 16 for r in recs[4:-3])
    back = dump.read_dump(str(tmp_path))
    assert (back.it, back.t, back.ndim, back.nx) == (12, t, ndim, p.nx)
    assert back.x0 == st.x0 > 0.0 and back.xlapse == st.xlapse > 0.0
    assert back.nptx == st.nptx and back.sptx_max == st.sptx_max
    assert np.array_equal(back.fields, st.fields)
    for a, b in zip(back.species, st.species):
        assert np.array_equal(a, b)
    assert np.array_equal(back.xpt, st.xpt) and np.array_equal(back.wghpt, st.wghpt)
    assert np.array_equal(back.ypt[0], st.ypt[0]) and np.array_equal(back.wghyz[0], st.wghyz[0])
    assert os.path.getsize(tmp_path / dump.FIELDS) == 8 * st.fields.size


@pytest.mark.parametrize("ndim", [2, 3])
def test_restart_continues_bit_exact(ndim, tmp_path):
    p, src, a = _fresh(ndim)
    t = _run(p, src, 12, holder=a)  # one window shift (iteration 10)
    dump.write_dump(str(tmp_path), dump.capture(a, p, 12, t, [src]), a.xmn() + (p.xmax - p.xmn))
    st = dump.read_dump(str(tmp_path))
    b = Oracle(dump.shifted_params(p, st.x0))
    b.set_plasma_source(src)
    dump.restore(b, st)
    assert b.xmn() == a.xmn()
    ta = _run(p, src, 12, t=t, it0=12, holder=a)  # through the shift and injection at 20
    tb = _run(p, src, 12, t=st.t, it0=st.it, holder=b)
    assert ta == tb
    assert np.array_equal(a.get_fields().view(np.uint64), b.get_fields().view(np.uint64))
    assert np.array_equal(a.get_species(0).view(np.uint64), b.get_species(0).view(np.uint64))
    assert a.window_state() == b.window_state()


def test_reference_dump_restarts_window_counters(tmp_path):
    p, src, a = _fresh(3)
    t = _run(p, src, 12, holder=a)
    st = dump.capture(a, p, 12, t, [src])
    st.xlapse = 0.0  # the reference does not write the window counter
    dump.write_dump(str(tmp_path), st, a.xmn() + (p.xmax - p.xmn))
    st = dump.read_dump(str(tmp_path))
    b = Oracle(dump.shifted_params(p, st.x0))
    b.set_plasma_source(src)
    dump.restore(b, st)
    t = st.t
    for it in range(12, 21):
        rc, out = b.lp_run(t, it)
        assert rc == 0
        t += p.dt
    # lp_window_xshift from xlapse = 0, wi1 = 0 at the first shift after the restart
    assert out.nshx == int(math.floor(p.dx_inv * p.w_speed * p.dt * p.w_sh + 0.5))


def test_dump_before_target_enters_window(tmp_path):
    """A dump taken while the box holds no particle yet (the target starts
    beyond the right edge) still carries the transverse lattice in
    Dist-wgyz.bin, as dump_data writes it whenever particles are part of the
    run (pic_dump.f90:336-377); the restart reads it and continues bit for
    bit through the window shift that brings the target in."""
    p = small_case(3, nx=40, ny=20, nz=12, cap=120_000)
    src = plasma_source(p)
    src.x_start = p.xmax + 3 * p.dx
    src.x_end = p.xmax + 40 * p.dx
    a = Oracle(p)
    a.set_fields(laser_fields(p))
    a.set_plasma_source(src)
    a.load_plasma(0)
    assert a.get_species(0).shape[0] == 0
    t = _run(p, src, 5, holder=a)
    st = dump.capture(a, p, 5, t, [src])
    dump.write_dump(str(tmp_path), st, a.xmn() + (p.xmax - p.xmn))
    assert not os.path.exists(tmp_path / dump.PARTICLES)
    assert os.path.getsize(tmp_path / dump.DISTYZ) == 8 * (len(st.ypt[0]) + len(st.zpt[0]) + st.wghyz[0].size) > 0
    back = dump.read_dump(str(tmp_path))
    assert back.ypt is not None and np.array_equal(back.ypt[0], st.ypt[0])
    assert np.array_equal(back.zpt[0], st.zpt[0]) and np.array_equal(back.wghyz[0], st.wghyz[0])
    b = Oracle(dump.shifted_params(p, back.x0))
    b.set_plasma_source(src)
    dump.restore(b, back)
    ta = _run(p, src, 19, t=t, it0=5, holder=a)  # through the shift at 10 (injection) and 20
    tb = _run(p, src, 19, t=back.t, it0=back.it, holder=b)
    assert ta == tb
    n = a.get_species(0).shape[0]
    assert n > 0 and b.get_species(0).shape[0] == n
    assert np.array_equal(a.get_species(0).view(np.uint64), b.get_species(0).view(np.uint64))
    assert np.array_equal(a.get_fields().view(np.uint64), b.get_fields().view(np.uint64))


# ---- dumps of several ranks (blocks of a y / z split) ---------------------------
def _block_states(p, lay, seed=4):
    from aladyn_b200.domain import SlabLayout  # noqa: F401  (layout type)
    rng = np.random.default_rng(seed)
    states = []
    ndv = 7 if p.ndim == 3 else 5
    nxpt = 30
    xpt = np.cumsum(rng.uniform(0.1, 0.2, (nxpt, 2)), axis=0)
    for r in range(lay.n):
        q = lay.params(r)
        n3p = q.nz + 5 if p.ndim == 3 else 1
        fields = np.asfortranarray(rng.standard_normal((q.nx + 5, q.ny + 5, n3p, p.nfield)))
        species = [np.asfortranarray(rng.standard_normal((int(rng.integers(0, 50)), ndv))) for _ in range(2)]
        ny_r = 2 * q.ny
        nz_r = 2 * q.nz if p.ndim == 3 else 1
        ypt = [np.linspace(q.gymin, q.gymax, ny_r), np.zeros(0)]
        zpt = [np.linspace(q.gzmin, q.gzmax, nz_r) if p.ndim == 3 else np.zeros(1), np.zeros(0)]
        wghyz = [rng.uniform(0.5, 1.5, (ny_r, nz_r)), np.zeros((0, 0))]
        states.append(dump.DumpState(it=17, t=3.25, ndim=p.ndim, nx=p.nx, fields=fields, species=species,
                                     nptx=[11, 0], sptx_max=[30, 0], x0=1.5, xlapse=1.4, ompe=p.ompe, targ_in=0.5,
                                     targ_end=1e3, xpt=xpt, wghpt=np.ones_like(xpt), ypt=ypt, zpt=zpt, wghyz=wghyz))
    return states


def _same_state(a, b):
    assert np.array_equal(a.fields, b.fields)
    assert len(a.species) == len(b.species)
    for x, y in zip(a.species, b.species):
        assert np.array_equal(x, y)
    for u, v in zip(a.ypt + a.zpt + a.wghyz, b.ypt + b.zpt + b.wghyz):
        assert np.array_equal(u, v)
    assert np.array_equal(a.xpt, b.xpt) and (a.it, a.t, a.x0, a.xlapse) == (b.it, b.t, b.x0, b.xlapse)
    assert list(a.nptx) == list(b.nptx) and list(a.sptx_max) == list(b.sptx_max)


@pytest.mark.parametrize("ndim,ny_s,nz_s", [(2, 2, 1), (3, 2, 2), (3, 1, 2)])
def test_block_dump_round_trip(ndim, ny_s, nz_s, tmp_path):
    """dump_data with npe_y x npe_z ranks: one EB-fields / Particles file per
    z column with the column's ranks in y order, Dist-wgyz in mype order,
    npt_arr(1:npe, 1:nsp) and dist_npy / dist_npz in Comm-data."""
    from aladyn_b200.domain import SlabLayout
    p = small_case(ndim, nx=16, ny=12, nz=8)
    lay = SlabLayout(p, ny_s, nz_s)
    states = _block_states(p, lay)
    d = str(tmp_path / "dump")
    dump.write_dump_blocks(d, states, lay, xmax=p.xmax)
    assert sorted(os.listdir(d)) == sorted(["Comm-data.bin", "Dist-wgyz.bin"] +
                                           [f"EB-fields{rz:02d}.bin" for rz in range(nz_s)] +
                                           [f"Particles{rz:02d}.bin" for rz in range(nz_s)])
    # rank imody of a column at imody times its length
    raw = np.fromfile(os.path.join(d, "EB-fields00.bin"))
    n = states[0].fields.size
    assert raw.size == ny_s * n and np.array_equal(raw[n:2 * n] if ny_s > 1 else raw[:n],
                                                   states[1 if ny_s > 1 else 0].fields.ravel(order="F"))
    back = dump.read_dump_blocks(d, lay)
    assert len(back) == lay.n
    for a, b in zip(states, back):
        _same_state(a, b)
    # the last three records of Comm-data: npt_arr(npe, nsp), dist_npy(npe_y, nsp), dist_npz(npe_z, nsp)
    data = open(os.path.join(d, "Comm-data.bin"), "rb").read()
    sizes = [4 * lay.n * 2, 4 * ny_s * 2, 4 * nz_s * 2]
    pos = len(data) - sum(s + 8 for s in sizes)
    npt = np.frombuffer(data[pos + 4:pos + 4 + sizes[0]], dtype=np.int32).reshape((lay.n, 2), order="F")
    assert npt.tolist() == [[st.species[ic].shape[0] for ic in range(2)] for st in states]


def test_block_dump_of_one_rank_is_the_single_rank_dump(tmp_path):
    from aladyn_b200.domain import SlabLayout
    p = small_case(3, nx=16, ny=12, nz=8)
    lay = SlabLayout(p, 1, 1)
    st = _block_states(p, lay)[0]
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    dump.write_dump(a, st, xmax=p.xmax)
    dump.write_dump_blocks(b, [st], lay, xmax=p.xmax)
    assert sorted(os.listdir(a)) == sorted(os.listdir(b))
    for name in os.listdir(a):
        assert open(os.path.join(a, name), "rb").read() == open(os.path.join(b, name), "rb").read(), name


def test_block_dump_needs_an_even_split(tmp_path):
    from aladyn_b200.domain import SlabLayout
    p = small_case(2, nx=16, ny=13)
    lay = SlabLayout(p, 2)
    with pytest.raises(ValueError):
        dump.write_dump_blocks(str(tmp_path / "d"), _block_states(p, lay), lay, xmax=p.xmax)
