"""Field and particle output in the reference's formats (fields_out and
part_pdata_out, src/IO/pic_out.f90:615-752, 1356-1500), for one rank and
for the ranks of a y / z split (the one-rank files byte-equal to a 1 x 1
split; several ranks' parts in mype order), from an oracle state: the .bin records read back to the sampled field and the
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


# ---- several ranks (blocks of a y / z split) -------------------------------------
def _split_state(ndim, ny_s, nz_s, jump_ok=True):
    from aladyn_b200.domain import SlabLayout
    p, o, t = _state(ndim)
    lay = SlabLayout(p, ny_s, nz_s)
    f = o.get_fields()
    part = o.get_species(0)
    fields = [lay.local(r, f) for r in range(lay.n)]
    parts = []
    for r in range(lay.n):
        q = lay.params(r)
        m = (part[:, 1] > q.gymin) & (part[:, 1] <= q.gymax)
        if ndim == 3:
            m &= (part[:, 2] > q.gzmin) & (part[:, 2] <= q.gzmax)
        parts.append(part[m])
    return p, lay, f, part, fields, parts, t


def test_block_writers_of_one_rank_equal_the_one_rank_files(tmp_path):
    p, lay, f, part, fields, parts, t = _split_state(3, 1, 1)
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    for jump in (1, 2):
        na = output.fields_out(a, p, f, 2, 2, 3, tnow=t, jump=jump)
        nb = output.fields_out_blocks(b, lay, fields, 2, 2, 3, tnow=t, jump=jump)
        for ext in (".bin", ".dat"):
            assert open(f"{a}/0003/{na}{ext}", "rb").read() == open(f"{b}/0003/{nb}{ext}", "rb").read()
    na = output.part_pdata_out(a, p, part, 1, 3, timenow=t, jmp=2, ymax_out=0.5 * p.gymax)
    nb = output.part_pdata_out_blocks(b, lay, parts, 1, 3, timenow=t, jmp=2, ymax_out=0.5 * p.gymax)
    for ext in (".bin", ".dat"):
        assert open(f"{a}/0003/{na}{ext}", "rb").read() == open(f"{b}/0003/{nb}{ext}", "rb").read()


@pytest.mark.parametrize("ndim,ny_s,nz_s", [(2, 2, 1), (3, 2, 2)])
def test_block_fields_and_particles_out(ndim, ny_s, nz_s, tmp_path):
    """npe ranks: after the parameters, each rank's gr_dim and its interior
    in mype order (together the whole interior), then the global grid; the
    particle file holds each rank's count and records one after the other."""
    from aladyn_b200.dump import read_records
    p, lay, f, part, fields, parts, t = _split_state(ndim, ny_s, nz_s)
    d = str(tmp_path)
    name = output.fields_out_blocks(d, lay, fields, 1, 1, 4, tnow=t)
    recs = read_records(f"{d}/0004/{name}.bin")
    assert len(recs) == 3 + 2 * lay.n + 3
    int_par = np.frombuffer(recs[1], dtype=np.int32)
    assert list(int_par[:3]) == [ny_s, nz_s, 1] and int_par[4] == p.ny
    assert int_par[6] == (p.nz if ndim == 3 else 1)
    nz = p.nz if ndim == 3 else 1
    glob = np.zeros((p.nx, p.ny, nz), dtype=np.float32)
    for r in range(lay.n):
        gr = np.frombuffer(recs[3 + 2 * r], dtype=np.int32)
        w = np.frombuffer(recs[4 + 2 * r], dtype=np.float32).reshape(tuple(gr), order="F")
        ry, rz = lay.coords(r)
        k0 = lay.k0[rz] if ndim == 3 else 0
        glob[:, lay.j0[ry]:lay.j0[ry] + gr[1], k0:k0 + gr[2]] = w
    ks = slice(2, p.nz + 2) if ndim == 3 else slice(0, 1)
    assert np.array_equal(glob, f[2:p.nx + 2, 2:p.ny + 2, ks, 0].astype(np.float32))
    pname = output.part_pdata_out_blocks(d, lay, parts, 1, 4, timenow=t)
    raw = open(f"{d}/0004/{pname}.bin", "rb").read()
    ndv = 2 * ndim + 2
    pos, total = 0, 0
    for r in range(lay.n):
        n = int(np.frombuffer(raw[pos:pos + 4], dtype=np.int32)[0])
        assert n == parts[r].shape[0]
        blk = np.frombuffer(raw[pos + 4:pos + 4 + 4 * n * ndv], dtype=np.float32).reshape((n, ndv))
        assert np.array_equal(blk[:, 0], parts[r][:, 0].astype(np.float32))
        pos += 4 + 4 * n * ndv
        total += n
    assert pos == len(raw) and total == part.shape[0]
    dat = open(f"{d}/0004/{pname}.dat").read()
    assert f"{total:20d}" in dat and f" npe =      {lay.n:8d}" in dat
