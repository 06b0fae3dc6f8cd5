"""Field and particle output files in the reference's formats: fields_out
and part_pdata_out (src/IO/pic_out.f90:615-752, 1356-1500) for one rank and,
``fields_out_blocks`` / ``part_pdata_out_blocks``, for the ranks of a y / z
split (every rank's part in mype order), written from any state holder's
arrays (the device's
``PicDevice.get_fields`` / ``get_species`` or the oracle's), so that the
reference's post-processing reads a run of this library.

Output directory ``%04d`` % iout.  Fields: for component f_ind, file
``<Ex|Ey|Ez|Bx|By|Bz|Jx>fout<iout>``:

``.dat``  formatted: `` Integer parameters`` then int_par(1:20) as
          ``(4i14)``, `` Real parameters`` then real_par(1:20) as
          ``(4e14.5)``;
``.bin``  Fortran unformatted sequential records: par_dim (= 20),
          int_par(20), real_par(20) (float32), gr_dim(3), the field sampled
          every ``jump`` interior node as float32 (x fastest), then the x, y
          and z grid coordinates sampled every ``jump`` (float32).

Particles of species pid (1-based), file ``<Elp|H1p|Prp|H2p>out<iout>``:

``.dat``  formatted: `` Real parameters`` and 20 lines ``(a13,e11.4)``,
          `` Integer parameters`` and 20 lines ``(a12,i8)``,
          `` Number of particles in the output box`` and the count ``(4i20)``;
``.bin``  stream (MPI-IO, one rank): int32 count, then per particle the
          nd2 phase-space coordinates, the weight and the charge as float32
          (records p = 1, 1 + jmp, ... inside the output box:
          xmin_out <= x <= xmax_out, |y| <= ymax_out [and |z| <= ymax_out]).

Namelist quantities the library does not hold (w0_x, a0, n_over_nc, ...)
come from the caller's ``run`` dictionary and default to 0.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

from .sim import unpack_slot

PAR_DIM = 20
FIELD_NAMES = {0: "Jxfout", 1: "Exfout", 2: "Eyfout", 4: "Bxfout", 5: "Byfout", 6: "Bzfout"}
PART_FILES = ["Elpout", "H1pout", "Prpout", "H2pout"]
RPAR = [" time =      ", " xmin =      ", " xmax =      ", " ymin =      ", " ymax =      ",
        " zmin =      ", " zmax =      ", " w0_x =      ", " w0_y =      ", " a0 =        ",
        " lam0 =      ", " mc2(MeV) =  ", " n0(e18) =   ", " np/cell =   ", " weight =    ",
        " mass =      ", " xmin_out =  ", " xmax_out =  ", " ymax_out =  ", " gam_min =   "]
IPAR = [" npe =      ", " nx =       ", " ny =       ", " nz =       ", " model =    ",
        " dmodel =   ", " nsp =      ", " curr_ndim =", " mp/cell =  ", " ion_ch =   ",
        " tsch_ord = ", " der_ord =  ", " iform =    ", " ph_sp_nc = ", " f_version =",
        " i_end =    ", " nx_loc =   ", " ny_loc =   ", " nz_loc =   ", " pjump  =   "]
ELECTRON_MASS = 0.510998928  # e0, src/work/phys_param.f90:47


def fortran_e(v: float, w: int, d: int) -> str:
    """Fortran Ew.d edit descriptor: [-]0.dddd E+xx, right-justified in w."""
    v = float(v)
    if v == 0.0:
        s = "0." + "0" * d + "E+00"
    else:
        e = math.floor(math.log10(abs(v))) + 1
        digits = int(round(abs(v) / 10.0 ** e * 10 ** d))
        if digits >= 10 ** d:  # rounded up to 1.000...: 0.1000 and the next exponent
            digits //= 10
            e += 1
        elif digits < 10 ** (d - 1):  # log10 rounding put the value one decade low
            digits = int(round(abs(v) / 10.0 ** (e - 1) * 10 ** d))
            e -= 1
        s = ("-" if v < 0 else "") + "0." + f"{digits:0{d}d}" + ("E+" if e >= 0 else "E-") + f"{abs(e):02d}"
    return s.rjust(w)


def _records(f, arrays):
    for a in arrays:
        b = np.ascontiguousarray(a).tobytes()
        n = np.array([len(b)], dtype=np.int32).tobytes()
        f.write(n + b + n)


def endian() -> int:
    """i_end of pic_out.f90:53-65: 1 on a little-endian host."""
    return 1 if sys.byteorder == "little" else 2


def _nsample(n: int, jump: int) -> int:
    return len(range(1, n + 1, jump))


def fields_out(dirpath: str, p, fields: np.ndarray, f_ind: int, f_var: int, iout: int, tnow: float = 0.0,
               jump: int = 1, run: dict | None = None, xmn: float | None = None) -> str:
    """One field component (f_ind, 1-based) of ebf(n1p, n2p, n3p, nf) as
    fields_out writes it; f_var names the file (1 Ex, 2 Ey, 3 Ez or Bz in 2D,
    4 Bx, 5 By, 6 Bz, 0 Jx).  Returns the file stem."""
    run = run or {}
    ndim = int(p.ndim)
    nx, ny, nz = int(p.nx), int(p.ny), int(p.nz) if ndim == 3 else 1
    x0 = p.xmn if xmn is None else xmn
    folder = os.path.join(dirpath, "%04d" % iout)
    os.makedirs(folder, exist_ok=True)
    name = FIELD_NAMES.get(f_var) or ("Bzfout" if p.nfield == 3 else "Ezfout")
    fname = "%s%02d" % (name, iout)
    ks = range(2, nz + 2, jump) if ndim == 3 else range(0, 1)
    sub = fields[2:nx + 2:jump, 2:ny + 2:jump, ks.start:ks.stop:jump if ndim == 3 else 1, f_ind - 1]
    wdata = np.asarray(sub, dtype=np.float32).ravel(order="F")
    gr_dim = np.array([_nsample(nx, jump), _nsample(ny, jump), _nsample(nz, jump) if ndim == 3 else 1], dtype=np.int32)
    int_par = np.array([1, 1, 1, gr_dim[0], gr_dim[1], ny, gr_dim[2], nz, jump, int(p.iby), int(p.iform),
                        run.get("model_id", 1), run.get("dmodel_id", 1), int(p.nsp), int(p.curr_ndim),
                        run.get("mp_per_cell", 0), run.get("lpf_ord", 2), run.get("der_ord", 2), 2, endian()],
                       dtype=np.int32)
    real_par = np.array([tnow, x0, x0 + nx * p.dx, p.gymin, p.gymax, p.gzmin, p.gzmax, run.get("w0_x", 0.0),
                         run.get("w0_y", 0.0), run.get("n_over_nc", 0.0), run.get("a0", 0.0), run.get("lam0", 0.0),
                         ELECTRON_MASS, p.ompe, run.get("targ_in", 0.0), run.get("targ_end", 0.0),
                         run.get("gam0", 0.0), run.get("nb_over_np", 0.0), run.get("b_charge", 0.0),
                         run.get("vbeam", 0.0)], dtype=np.float32)
    with open(os.path.join(folder, fname + ".dat"), "w") as f:
        f.write("  Integer parameters\n")
        for r in range(0, PAR_DIM, 4):
            f.write("".join(f"{int(v):14d}" for v in int_par[r:r + 4]) + "\n")
        f.write("  Real parameters\n")
        for r in range(0, PAR_DIM, 4):
            f.write("".join(fortran_e(v, 14, 5) for v in real_par[r:r + 4]) + "\n")
    xg = (x0 + p.dx * np.arange(0, nx, jump)).astype(np.float32)
    yg = (p.dy * (np.arange(1, ny + 1, jump) - 1 - ny // 2)).astype(np.float32)
    zg = (p.dz * (np.arange(1, nz + 1, jump) - 1 - nz // 2)).astype(np.float32) if ndim == 3 else \
        np.zeros(1, dtype=np.float32)
    with open(os.path.join(folder, fname + ".bin"), "wb") as f:
        _records(f, [np.array([PAR_DIM], dtype=np.int32), int_par, real_par, gr_dim, wdata, xg, yg, zg])
    return fname


def _pdata(p, part: np.ndarray, jmp: int, xmin_out: float, xmax_out: float, ymax_out: float) -> np.ndarray:
    """The output records (float32: phase space, weight, charge) of records
    p = 1, 1 + jmp, ... inside the output box."""
    ndim = int(p.ndim)
    nd2 = 2 * ndim
    sel = part[::jmp]
    keep = (np.abs(sel[:, 1]) <= ymax_out)
    if ndim == 3:
        keep &= np.abs(sel[:, 2]) <= ymax_out
    keep &= (sel[:, 0] >= xmin_out) & (sel[:, 0] <= xmax_out)
    sel = sel[keep]
    charge, _, wgh = unpack_slot(sel[:, nd2])
    pdata = np.empty((sel.shape[0], nd2 + 2), dtype=np.float32)
    pdata[:, :nd2] = sel[:, :nd2].astype(np.float32)
    pdata[:, nd2] = wgh
    pdata[:, nd2 + 1] = charge.astype(np.float32)
    return pdata


def _part_pars(p, pid, timenow, x0, xmin_out, xmax_out, ymax_out, jmp, run, npe, loc):
    ndim = int(p.ndim)
    ndv = 2 * ndim + 2
    nx, ny, nz = int(p.nx), int(p.ny), int(p.nz) if ndim == 3 else 1
    real_par = np.array([timenow, x0, x0 + nx * p.dx, p.gymin, p.gymax, p.gzmin, p.gzmax, run.get("w0_x", 0.0),
                         run.get("w0_y", 0.0), run.get("a0", 0.0), run.get("lam0", 0.0), ELECTRON_MASS,
                         run.get("n0_ref", 0.0), run.get("np_per_cell", 0.0), run.get("j0_norm", 0.0),
                         1.0 / p.lorentz_fact[pid - 1], xmin_out, xmax_out, ymax_out, run.get("gam_min", 0.0)],
                        dtype=np.float32)
    int_par = np.array([npe, nx, ny, nz, run.get("model_id", 1), run.get("dmodel_id", 1), int(p.nsp),
                        int(p.curr_ndim), run.get("mp_per_cell", 0), run.get("ion_min", 0), run.get("lpf_ord", 2),
                        run.get("der_ord", 2), int(p.iform), ndv, 4, endian(), loc[0], loc[1], loc[2], jmp],
                       dtype=np.int32)
    return real_par, int_par


def _write_part(folder, fname, real_par, int_par, pdatas):
    ip = sum(d.shape[0] for d in pdatas)
    with open(os.path.join(folder, fname + ".dat"), "w") as f:
        f.write("  Real parameters\n")
        for q in range(PAR_DIM):
            f.write(RPAR[q] + fortran_e(real_par[q], 11, 4) + "\n")
        f.write("  Integer parameters\n")
        for q in range(PAR_DIM):
            f.write(IPAR[q] + f"{int(int_par[q]):8d}\n")
        f.write("  Number of particles in the output box\n")
        f.write(f"{ip:20d}\n")
    # each rank at mype + ndv * (records of the ranks before it), 4-byte
    # units: its count, then its records
    with open(os.path.join(folder, fname + ".bin"), "wb") as f:
        for d in pdatas:
            f.write(np.array([d.shape[0]], dtype=np.int32).tobytes())
            f.write(d.tobytes())


def part_pdata_out(dirpath: str, p, part: np.ndarray, pid: int, iout: int, timenow: float = 0.0,
                   xmin_out: float = -1e30, xmax_out: float = 1e30, ymax_out: float = 1e30, jmp: int = 1,
                   run: dict | None = None, xmn: float | None = None) -> str:
    """Species pid (1-based) records part(np, ndv) as part_pdata_out writes
    them.  Returns the file stem."""
    run = run or {}
    x0 = p.xmn if xmn is None else xmn
    folder = os.path.join(dirpath, "%04d" % iout)
    os.makedirs(folder, exist_ok=True)
    pdata = _pdata(p, part, jmp, xmin_out, xmax_out, ymax_out)
    nz = int(p.nz) if p.ndim == 3 else 1
    real_par, int_par = _part_pars(p, pid, timenow, x0, xmin_out, xmax_out, ymax_out, jmp, run, 1,
                                   (int(p.nx), int(p.ny), nz))
    fname = "%s%02d" % (PART_FILES[pid - 1], iout)
    _write_part(folder, fname, real_par, int_par, [pdata])
    return fname


def part_pdata_out_blocks(dirpath: str, layout, parts, pid: int, iout: int, timenow: float = 0.0,
                          xmin_out: float = -1e30, xmax_out: float = 1e30, ymax_out: float = 1e30, jmp: int = 1,
                          run: dict | None = None, xmn: float | None = None) -> str:
    """part_pdata_out of a run split into blocks (``parts[r]`` of block r,
    mype order): one file, each rank's count and records one after the
    other; npe and the first rank's local sizes in the parameters."""
    run = run or {}
    p = layout.p
    x0 = p.xmn if xmn is None else xmn
    folder = os.path.join(dirpath, "%04d" % iout)
    os.makedirs(folder, exist_ok=True)
    pdatas = [_pdata(layout.params(r), parts[r], jmp, xmin_out, xmax_out, ymax_out) for r in range(layout.n)]
    q0 = layout.params(0)
    real_par, int_par = _part_pars(p, pid, timenow, x0, xmin_out, xmax_out, ymax_out, jmp, run, layout.n,
                                   (int(q0.nx), int(q0.ny), int(q0.nz) if p.ndim == 3 else 1))
    fname = "%s%02d" % (PART_FILES[pid - 1], iout)
    _write_part(folder, fname, real_par, int_par, pdatas)
    return fname


def fields_out_blocks(dirpath: str, layout, fields, f_ind: int, f_var: int, iout: int, tnow: float = 0.0,
                      jump: int = 1, run: dict | None = None, xmn: float | None = None) -> str:
    """fields_out of a run split into blocks (``fields[r]``, the local
    ebf of block r, mype order): rank 0 writes the parameters, then each
    rank's gr_dim and its interior sampled every ``jump`` node from its own
    first node, in mype order, then the global grid coordinates; int_par
    starts with npe_y, npe_z, npe_x and the summed sample counts."""
    run = run or {}
    p = layout.p
    ndim = int(p.ndim)
    nx, ny, nz = int(p.nx), int(p.ny), int(p.nz) if ndim == 3 else 1
    x0 = p.xmn if xmn is None else xmn
    folder = os.path.join(dirpath, "%04d" % iout)
    os.makedirs(folder, exist_ok=True)
    name = FIELD_NAMES.get(f_var) or ("Bzfout" if p.nfield == 3 else "Ezfout")
    fname = "%s%02d" % (name, iout)
    blocks = []
    for r in range(layout.n):
        q = layout.params(r)
        qny, qnz = int(q.ny), int(q.nz) if ndim == 3 else 1
        f = fields[r]
        sub = f[2:nx + 2:jump, 2:qny + 2:jump, 2:qnz + 2:jump if ndim == 3 else 1, f_ind - 1] if ndim == 3 \
            else f[2:nx + 2:jump, 2:qny + 2:jump, 0:1, f_ind - 1]
        gr = np.array([_nsample(nx, jump), _nsample(qny, jump), _nsample(qnz, jump) if ndim == 3 else 1],
                      dtype=np.int32)
        blocks.append((gr, np.asarray(sub, dtype=np.float32).ravel(order="F")))
    nyh = [_nsample(layout.rows[ry], jump) for ry in range(layout.ny_s)]
    nzh = [_nsample(layout.planes[rz], jump) for rz in range(layout.nz_s)] if ndim == 3 else [1]
    int_par = np.array([layout.ny_s, layout.nz_s, 1, _nsample(nx, jump), sum(nyh), max(layout.rows),
                        sum(nzh), max(layout.planes) if ndim == 3 else 1, jump, int(p.iby), int(p.iform),
                        run.get("model_id", 1), run.get("dmodel_id", 1), int(p.nsp), int(p.curr_ndim),
                        run.get("mp_per_cell", 0), run.get("lpf_ord", 2), run.get("der_ord", 2), 2, endian()],
                       dtype=np.int32)
    real_par = np.array([tnow, x0, x0 + nx * p.dx, p.gymin, p.gymax, p.gzmin, p.gzmax, run.get("w0_x", 0.0),
                         run.get("w0_y", 0.0), run.get("n_over_nc", 0.0), run.get("a0", 0.0), run.get("lam0", 0.0),
                         ELECTRON_MASS, p.ompe, run.get("targ_in", 0.0), run.get("targ_end", 0.0),
                         run.get("gam0", 0.0), run.get("nb_over_np", 0.0), run.get("b_charge", 0.0),
                         run.get("vbeam", 0.0)], dtype=np.float32)
    with open(os.path.join(folder, fname + ".dat"), "w") as f:
        f.write("  Integer parameters\n")
        for r in range(0, PAR_DIM, 4):
            f.write("".join(f"{int(v):14d}" for v in int_par[r:r + 4]) + "\n")
        f.write("  Real parameters\n")
        for r in range(0, PAR_DIM, 4):
            f.write("".join(fortran_e(v, 14, 5) for v in real_par[r:r + 4]) + "\n")
    xg = (x0 + p.dx * np.arange(0, nx, jump)).astype(np.float32)
    yg = (p.dy * (np.arange(1, ny + 1, jump) - 1 - ny // 2)).astype(np.float32)
    zg = (p.dz * (np.arange(1, nz + 1, jump) - 1 - nz // 2)).astype(np.float32) if ndim == 3 else \
        np.zeros(1, dtype=np.float32)
    recs = [np.array([PAR_DIM], dtype=np.int32), int_par, real_par]
    for gr, w in blocks:
        recs += [gr, w]
    with open(os.path.join(folder, fname + ".bin"), "wb") as f:
        _records(f, recs + [xg, yg, zg])
    return fname


# ---- readers ----------------------------------------------------------------
def read_fields_bin(path: str):
    """(int_par, real_par, gr_dim, field(nx, ny, nz) float32, x, y, z) of a
    fields_out .bin file."""
    from .dump import read_records
    recs = read_records(path)
    if np.frombuffer(recs[0], dtype=np.int32)[0] != PAR_DIM:
        raise ValueError(f"{path}: par_dim record")
    int_par = np.frombuffer(recs[1], dtype=np.int32)
    real_par = np.frombuffer(recs[2], dtype=np.float32)
    gr_dim = np.frombuffer(recs[3], dtype=np.int32)
    data = np.frombuffer(recs[4], dtype=np.float32).reshape(tuple(gr_dim), order="F")
    return (int_par, real_par, gr_dim, data, np.frombuffer(recs[5], dtype=np.float32),
            np.frombuffer(recs[6], dtype=np.float32), np.frombuffer(recs[7], dtype=np.float32))


def read_part_bin(path: str, ndv: int) -> np.ndarray:
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:4], dtype=np.int32)[0])
    return np.frombuffer(raw[4:], dtype=np.float32).reshape((n, ndv))
