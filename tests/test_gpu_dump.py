"""Dump / restart of the device state (aladyn_b200.dump with PicDevice):
a run in the FP64 form's deterministic mode dumped after a window shift and
restarted in a new handle continues bit for bit like the uninterrupted run,
through the next window shift and injection; the split form restarts to
its own FP32 round-off."""
import numpy as np
import pytest

from aladyn_b200 import dump
from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.sim import PicDevice
from tests.helpers import laser_fields, plasma_source, small_case

pytestmark = pytest.mark.gpu


def _fresh(ndim, precision):
    p = small_case(ndim, precision=precision, nx=40, ny=20, nz=12, cap=120_000)
    src = plasma_source(p)
    src.x_end = p.xmax + 40 * p.dx
    d = PicDevice(p)
    d.set_fields(laser_fields(p))
    d.set_plasma_source(src)
    d.load_plasma(0)
    return p, src, d


def _run(d, p, t, it0, steps, det):
    for it in range(it0, it0 + steps):
        out = d.lp_run(t, it, initial_time=(it == 0))
        assert out.error_bits == 0
        t += p.dt
    return t


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("precision", [AGPU_FP64, AGPU_FP32_SPLIT])
def test_device_restart(ndim, precision, tmp_path):
    det = precision == AGPU_FP64
    p, src, a = _fresh(ndim, precision)
    if det:
        a.set_deterministic(True)
    t = _run(a, p, 0.0, 0, 12, det)
    st = dump.capture(a, p, 12, t, [src])
    dump.write_dump(str(tmp_path), st, st.x0 + p.xmax)
    st = dump.read_dump(str(tmp_path))
    b = PicDevice(dump.shifted_params(p, st.x0))
    if det:
        b.set_deterministic(True)
    b.set_plasma_source(src)
    dump.restore(b, st)
    assert b.window_state() == a.window_state()
    _run(a, p, t, 12, 12, det)
    _run(b, p, st.t, st.it, 12, det)
    fa, fb = a.get_fields(), b.get_fields()
    sa, sb = a.get_species(0), b.get_species(0)
    assert a.window_state() == b.window_state()
    if det:
        assert np.array_equal(fa.view(np.uint64), fb.view(np.uint64))
        assert np.array_equal(sa.view(np.uint64), sb.view(np.uint64))
    else:
        assert sa.shape == sb.shape
        assert np.abs(fa - fb).max() <= 1e-4 * np.abs(fa).max()


def test_block_restart_bitexact(tmp_path):
    """2 x 2 blocks of a y / z split (FP64, deterministic mode) dumped as
    npe = 4 ranks after 6 steps (write_dump_blocks: the reference's files for
    several ranks), read back into four new handles, and run on through a
    window shift with injection: every block's fields and records equal the
    uninterrupted blocks' bit for bit."""
    from aladyn_b200.domain import Slab, SlabLayout, ThreadExchanger, run_threads
    p = small_case(3, w_sh=10)
    lay = SlabLayout(p, 2, 2)
    src = plasma_source(p, x_start_frac=0.3)
    ebf = laser_fields(p)

    def blocks():
        ex = ThreadExchanger(lay.n)
        out = []
        for r in range(lay.n):
            dev = PicDevice(lay.params(r))
            dev.set_plasma_source(src)
            dev.set_deterministic(True)
            out.append(Slab(lay, r, dev, ex))
        return out

    def steps(bl, it0, n):
        shifts = 0
        for it in range(it0, it0 + n):
            outs = [None] * lay.n

            def one(s):
                outs[s.rank] = s.dev.lp_run(it * p.dt, it, initial_time=(it == 0))

            run_threads(bl, one)
            assert all(o.error_bits == 0 for o in outs)
            shifts += outs[0].nshx > 0
        return outs, shifts

    a = blocks()
    for s in a:
        s.dev.set_fields(lay.local(s.rank, ebf))
        s.dev.load_plasma(0)
    steps(a, 0, 6)
    states = [dump.capture(s.dev, lay.params(s.rank), 6, 6 * p.dt, sources=[src]) for s in a]
    d = str(tmp_path / "dumpRestart")
    dump.write_dump_blocks(d, states, lay, xmax=p.xmax)
    b = blocks()
    for s, st in zip(b, dump.read_dump_blocks(d, lay)):
        dump.restore(s.dev, st)
    oa, sha = steps(a, 6, 6)
    ob, shb = steps(b, 6, 6)
    assert sha == shb == 1
    for sa, sb, x, y in zip(a, b, oa, ob):
        assert x.np[0] == y.np[0]
        assert np.array_equal(sa.dev.get_fields(), sb.dev.get_fields())
        ra, rb = sa.dev.get_species(0), sb.dev.get_species(0)
        assert np.array_equal(ra.view(np.uint64), rb.view(np.uint64))
