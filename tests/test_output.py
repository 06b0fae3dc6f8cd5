"""Field and particle output in the reference's formats (fields_out and
part_pdata_out, src/IO/pic_out.f90:615-752, 1356-1500), one rank, from an
oracle state: the .bin records read back to the sampled field and the
selected particle records (float32), the headers carry the grid sizes, the
sampling jump, the endianness flag and the box, and the .dat files hold
the parameters in the Fortran edit formats."""
import numpy as np
import pytest

from aladyn_b200 import output
from aladyn_b200.sim import unpack_slot
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case


def _state(ndim):
    p = small_case(ndim, nx=40, ny=20, nz=12, cap=120_000)
    o = Oracle(p)
    o.set_fields(laser_fields(p))
    o.set_plasma_source(plasma_source(p))
    o.load_plasma(0)
    t = 0.0
    for it in range(12):  # a window shift at step 10
        o.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    return p, o, t


def test_fortran_e_format():
    assert output.fortran_e(12.345, 14, 5) == "   0.12345E+02"
    assert output.fortran_e(-0.00123456, 11, 4) == "-0.1235E-02"
    assert output.fortran_e(0.0, 14, 5) == "   0.00000E+00"
    assert output.fortran_e(9.99999, 14, 5) == "   0.10000E+02"
    assert output.fortran_e(1.0, 11, 4) == " 0.1000E+01"


@pytest.mark.parametrize("ndim,jump", [(3, 1), (3, 2), (2, 3)])
def test_fields_out_round_trip(ndim, jump, tmp_path):
    p, o, t = _state(ndim)
    f = o.get_fields()
    xmn = o.xmn()
    stem = output.fields_out(str(tmp_path), p, f, 2, 2, 7, tnow=t, jump=jump, run={"a0": 2.0, "lam0": 0.8}, xmn=xmn)
    assert stem == "Eyfout07"
    ip, rp, gd, data, x, y, z = output.read_fields_bin(str(tmp_path / "0007" / (stem + ".bin")))
    ks = slice(2, p.nz + 2, jump) if ndim == 3 else slice(0, 1)
    expect = f[2:p.nx + 2:jump, 2:p.ny + 2:jump, ks, 1].astype(np.float32)
    assert tuple(gd) == expect.shape and np.array_equal(data, expect)
    assert ip[8] == jump and ip[3] == gd[0] and ip[4] == gd[1] and ip[19] == output.endian()
    assert rp[0] == np.float32(t) and rp[1] == np.float32(xmn) and rp[10] == np.float32(2.0)
    assert x.shape == (gd[0],) and x[0] == np.float32(xmn) and np.allclose(np.diff(x), jump * p.dx, rtol=1e-5)
    assert y.shape == (gd[1],) and np.isclose(y[0], p.ymn, rtol=1e-6)
    lines = open(tmp_path / "0007" / (stem + ".dat")).read().splitlines()
    assert lines[0].strip() == "Integer parameters" and lines[6].strip() == "Real parameters"
    assert [int(v) for v in lines[1].split()] == list(ip[:4])
    assert np.allclose([float(v) for v in lines[7].split()], rp[:4], rtol=6e-5)  # five digits


@pytest.mark.parametrize("ndim", [2, 3])
def test_part_pdata_out_round_trip(ndim, tmp_path):
    p, o, t = _state(ndim)
    part = o.get_species(0)
    xmin_out = part[:, 0].min() + 0.3 * np.ptp(part[:, 0])
    ymax_out = 0.4 * p.gymax
    stem = output.part_pdata_out(str(tmp_path), p, part, 1, 3, timenow=t, xmin_out=xmin_out, ymax_out=ymax_out,
                                 jmp=2, xmn=o.xmn())
    assert stem == "Elpout03"
    ndv = 2 * ndim + 2
    got = output.read_part_bin(str(tmp_path / "0003" / (stem + ".bin")), ndv)
    sel = part[::2]
    keep = (np.abs(sel[:, 1]) <= ymax_out) & (sel[:, 0] >= xmin_out)
    if ndim == 3:
        keep &= np.abs(sel[:, 2]) <= ymax_out
    sel = sel[keep]
    assert 0 < got.shape[0] == sel.shape[0] < part.shape[0]
    assert np.array_equal(got[:, :2 * ndim], sel[:, :2 * ndim].astype(np.float32))
    q, _, w = unpack_slot(sel[:, -1])
    assert np.array_equal(got[:, -2], w) and np.array_equal(got[:, -1], q.astype(np.float32))
    dat = open(tmp_path / "0003" / (stem + ".dat")).read().splitlines()
    assert dat[0].strip() == "Real parameters" and dat[21].strip() == "Integer parameters"
    assert dat[42].strip() == "Number of particles in the output box" and int(dat[43]) == got.shape[0]
    assert dat[1].startswith(" time =") and dat[22].startswith(" npe =") and int(dat[35].split()[-1]) == ndv
