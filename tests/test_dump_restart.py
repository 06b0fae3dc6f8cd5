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
