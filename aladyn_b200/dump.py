"""Dump and restart in the reference's ``dumpRestart/`` file formats
(``dump_data`` / ``restart``, src/start/pic_dump.f90:35-380, 382-795): a run
of this library can be continued by the reference and a reference dump can
be continued here, for one rank (``write_dump`` / ``read_dump``) or for the
blocks of a y / z split (``write_dump_blocks`` / ``read_dump_blocks``, npe_y
x npe_z ranks; no envelope or fluid arrays, which this library does not
evolve on blocks).

Files of a dump directory:

``Comm-data.bin``
    Fortran unformatted sequential records (4-byte length markers before and
    after each record; default integers of 4 bytes, reals of 8 bytes):

    * ``rdata(1:10)``: t, j0_norm, ompe, targ_in, targ_end, lp_in(1),
      xp0_out, xp1_out, x(1) (the distance the window has moved the box),
      rdata(10) (not read by the reference; here the window counter xlapse,
      0 in the reference's dumps);
    * ``ndata(1:10)``: iter, n1p, n2p, n3p, nptx_max, size(x) = nx + 2,
      nxf (0), nd2, 0, 0;
    * ``nptx(1:nsp)``, ``sptx_max(1:nsp)``;
    * when targ_end > xmax: nsp * nptx_max records ``(xpt(j, ic), wghpt(j, ic))``,
      j fastest;
    * ``npt_arr(1, 1:nsp)``, ``dist_npy(1, 1:nsp)``, ``dist_npz(1, 1:nsp)``.

``EB-fields00.bin``
    ``ebf(1:n1p, 1:n2p, 1:n3p, 1:nf)``, raw FP64 in Fortran order.
``Particles00.bin``
    for each species holding particles, ``spec(ic)%part(1:np, 1:ndv)`` raw
    FP64 column by column (written only when some species holds particles).
``Dist-wgyz.bin``
    ``loc_ypt(1:npty, ic)`` per species, ``loc_zpt(1:nptz, ic)`` per species,
    ``loc_wghyz(1:npty, 1:nptz, ic)`` per species, raw FP64 (written
    whenever the run has particle species, even before any particle is in
    the box, and read whenever present).

The (iter, t) of a dump are those of the next step, as the reference's main
loop writes them after ``timing`` (src/ALaDyn.F90:92-106).  A restart builds
its parameters with the box moved by x(1) (``shifted_params``, as restart
shifts x, xmin, xmax and the grid bounds, pic_dump.f90:515-526), then sets
the plasma sources, fields and particles, and the window state (xlapse,
nptx).  With xlapse 0, as in the reference's own dumps, the window counters
restart from zero as they do in the reference.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional

import numpy as np

COMM = "Comm-data.bin"
# one (xpt, wghpt) record of Comm-data.bin with its length markers
XPT_RECORD = np.dtype([("n0", "<i4"), ("x", "<f8"), ("w", "<f8"), ("n1", "<i4")])
XPT_MAX_COLUMNS = 1 << 26
FIELDS = "EB-fields00.bin"
PARTICLES = "Particles00.bin"
DISTYZ = "Dist-wgyz.bin"


# ---- Fortran unformatted sequential records -------------------------------
def write_records(path: str, records) -> None:
    with open(path, "wb") as f:
        for r in records:
            b = np.ascontiguousarray(r).tobytes()
            n = np.array([len(b)], dtype=np.int32).tobytes()
            f.write(n)
            f.write(b)
            f.write(n)


def read_records(path: str) -> List[bytes]:
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        if pos + 4 > len(data):
            raise ValueError(f"{path}: truncated record marker at byte {pos}")
        n = int(np.frombuffer(data, dtype=np.int32, count=1, offset=pos)[0])
        if n < 0 or pos + 8 + n > len(data):
            raise ValueError(f"{path}: bad record length {n} at byte {pos}")
        body = data[pos + 4:pos + 4 + n]
        tail = int(np.frombuffer(data, dtype=np.int32, count=1, offset=pos + 4 + n)[0])
        if tail != n:
            raise ValueError(f"{path}: record markers {n} and {tail} differ at byte {pos}")
        out.append(body)
        pos += n + 8
    return out


@dataclasses.dataclass
class DumpState:
    """What a dump holds for one rank."""
    it: int
    t: float
    ndim: int
    nx: int
    fields: np.ndarray                     # ebf(n1p, n2p, n3p, nf), Fortran order
    species: List[np.ndarray]              # part(np, ndv) per species (nsp entries)
    nptx: List[int]                        # lattice columns already injected
    sptx_max: List[int]                    # last column inside the target
    x0: float = 0.0                        # x(1): distance the window moved the box
    xlapse: float = 0.0                    # window counter (rdata(10))
    j0_norm: float = 0.0
    ompe: float = 0.0
    targ_in: float = 0.0
    targ_end: float = 0.0
    lp_in: float = 0.0
    xp0_out: float = 0.0
    xp1_out: float = 0.0
    xpt: Optional[np.ndarray] = None       # (nptx_max, nsp), written when targ_end > xmax
    wghpt: Optional[np.ndarray] = None
    ypt: Optional[List[np.ndarray]] = None  # per species, transverse lattice
    zpt: Optional[List[np.ndarray]] = None
    wghyz: Optional[List[np.ndarray]] = None  # per species, (npty, nptz)

    @property
    def nsp(self) -> int:
        return len(self.species)


def write_dump(dirpath: str, st: DumpState, xmax: float) -> None:
    """Write ``st`` as the reference's dumpRestart files into ``dirpath``;
    ``xmax`` is the current right end of the box (the xpt table is written
    when the target extends beyond it, as dump_data does)."""
    os.makedirs(dirpath, exist_ok=True)
    nsp = st.nsp
    n1p, n2p, n3p = st.fields.shape[:3]
    nd2 = 2 * st.ndim
    with_xpt = st.targ_end > xmax
    nptx_max = 0 if st.xpt is None else st.xpt.shape[0]
    if with_xpt and st.xpt is None:
        raise ValueError("targ_end > xmax: the dump needs the xpt / wghpt table")
    rdata = np.array([st.t, st.j0_norm, st.ompe, st.targ_in, st.targ_end, st.lp_in, st.xp0_out, st.xp1_out, st.x0,
                      st.xlapse], dtype=np.float64)
    ndata = np.array([st.it, n1p, n2p, n3p, nptx_max, st.nx + 2, 0, nd2, 0, 0], dtype=np.int32)
    head = [rdata, ndata, np.asarray(st.nptx, dtype=np.int32), np.asarray(st.sptx_max, dtype=np.int32)]
    npty = [0 if st.ypt is None else len(st.ypt[ic]) for ic in range(nsp)]
    nptz = [0 if st.zpt is None else len(st.zpt[ic]) for ic in range(nsp)]
    tail = [np.array([s.shape[0] for s in st.species], dtype=np.int32), np.asarray(npty, dtype=np.int32),
            np.asarray(nptz, dtype=np.int32)]
    path = os.path.join(dirpath, COMM)
    write_records(path, head)
    if with_xpt:
        # nsp * nptx_max records of (xpt, wghpt), j fastest, in one block
        blk = np.zeros(nsp * nptx_max, dtype=XPT_RECORD)
        blk["n0"] = 16
        blk["n1"] = 16
        blk["x"] = np.asarray(st.xpt, dtype=np.float64).T.ravel()
        blk["w"] = np.asarray(st.wghpt, dtype=np.float64).T.ravel()
        with open(path, "ab") as f:
            f.write(blk.tobytes())
    with open(path, "ab") as f:
        for r in tail:
            b = np.ascontiguousarray(r).tobytes()
            n = np.array([len(b)], dtype=np.int32).tobytes()
            f.write(n + b + n)
    np.asfortranarray(st.fields, dtype=np.float64).ravel(order="F").tofile(os.path.join(dirpath, FIELDS))
    if any(s.shape[0] > 0 for s in st.species):
        with open(os.path.join(dirpath, PARTICLES), "wb") as f:
            for s in st.species:
                if s.shape[0] > 0:
                    np.asarray(s, dtype=np.float64).ravel(order="F").tofile(f)
    # dump_data writes the transverse lattice whenever particles are part of
    # the run, even with no particle in the box yet (a dump taken before the
    # target enters the window), and restart reads it unconditionally
    # (pic_dump.f90:336-377, 733-760)
    if nsp > 0:
        with open(os.path.join(dirpath, DISTYZ), "wb") as f:
            for ic in range(nsp):
                if npty[ic] > 0:
                    np.asarray(st.ypt[ic], dtype=np.float64).tofile(f)
            for ic in range(nsp):
                if nptz[ic] > 0:
                    np.asarray(st.zpt[ic], dtype=np.float64).tofile(f)
            for ic in range(nsp):
                if nptz[ic] > 0 and npty[ic] > 0:
                    np.asarray(st.wghyz[ic], dtype=np.float64).ravel(order="F").tofile(f)


def _records_at(data: bytes, pos: int, count: int, path: str):
    out = []
    for _ in range(count):
        if pos + 4 > len(data):
            raise ValueError(f"{path}: truncated record marker at byte {pos}")
        n = int(np.frombuffer(data, dtype=np.int32, count=1, offset=pos)[0])
        if n < 0 or pos + 8 + n > len(data):
            raise ValueError(f"{path}: bad record length {n} at byte {pos}")
        if int(np.frombuffer(data, dtype=np.int32, count=1, offset=pos + 4 + n)[0]) != n:
            raise ValueError(f"{path}: record markers differ at byte {pos}")
        out.append(data[pos + 4:pos + 4 + n])
        pos += n + 8
    return out, pos


def read_dump(dirpath: str) -> DumpState:
    """Read a dumpRestart directory written by the reference (one rank) or by
    ``write_dump``."""
    path = os.path.join(dirpath, COMM)
    with open(path, "rb") as f:
        data = f.read()
    head, pos = _records_at(data, 0, 4, path)
    rdata = np.frombuffer(head[0], dtype=np.float64)
    ndata = np.frombuffer(head[1], dtype=np.int32)
    if rdata.size != 10 or ndata.size != 10:
        raise ValueError(f"{path}: rdata / ndata records of {rdata.size} / {ndata.size} values")
    nptx = np.frombuffer(head[2], dtype=np.int32).astype(int).tolist()
    sptx_max = np.frombuffer(head[3], dtype=np.int32).astype(int).tolist()
    nsp = len(nptx)
    it, n1p, n2p, n3p, nptx_max, nx2, _, nd2 = (int(v) for v in ndata[:8])
    ndim = nd2 // 2
    tail_bytes = 3 * (8 + 4 * nsp) + 0
    xpt = wghpt = None
    nblk = len(data) - pos - tail_bytes
    if nblk > 0:
        # the (xpt, wghpt) records (written when the target reaches beyond the box)
        if nblk != nsp * nptx_max * XPT_RECORD.itemsize:
            raise ValueError(f"{path}: {nblk} bytes of xpt records, expected {nsp * nptx_max} records")
        blk = np.frombuffer(data, dtype=XPT_RECORD, count=nsp * nptx_max, offset=pos)
        if np.any(blk["n0"] != 16) or np.any(blk["n1"] != 16):
            raise ValueError(f"{path}: bad xpt record markers")
        xpt = np.ascontiguousarray(blk["x"].reshape(nsp, nptx_max).T)
        wghpt = np.ascontiguousarray(blk["w"].reshape(nsp, nptx_max).T)
        pos += nblk
    recs, pos = _records_at(data, pos, 3, path)
    if pos != len(data):
        raise ValueError(f"{path}: {len(data) - pos} bytes after the last record")
    npt = np.frombuffer(recs[0], dtype=np.int32).astype(int).tolist()
    npty = np.frombuffer(recs[1], dtype=np.int32).astype(int).tolist()
    nptz = np.frombuffer(recs[2], dtype=np.int32).astype(int).tolist()
    raw = np.fromfile(os.path.join(dirpath, FIELDS), dtype=np.float64)
    ncell = n1p * n2p * n3p
    if raw.size % ncell:
        raise ValueError(f"{dirpath}/{FIELDS}: {raw.size} values, not a multiple of {ncell}")
    fields = raw.reshape((n1p, n2p, n3p, raw.size // ncell), order="F")
    ndv = nd2 + 1
    species = []
    if sum(npt) > 0:
        praw = np.fromfile(os.path.join(dirpath, PARTICLES), dtype=np.float64)
        if praw.size != ndv * sum(npt):
            raise ValueError(f"{dirpath}/{PARTICLES}: {praw.size} values, expected {ndv * sum(npt)}")
        off = 0
        for n in npt:
            species.append(praw[off:off + n * ndv].reshape((n, ndv), order="F").copy(order="F"))
            off += n * ndv
    else:
        species = [np.zeros((0, ndv), order="F") for _ in range(nsp)]
    ypt = zpt = wghyz = None
    if os.path.exists(os.path.join(dirpath, DISTYZ)):
        d = np.fromfile(os.path.join(dirpath, DISTYZ), dtype=np.float64)
        off = 0
        ypt, zpt, wghyz = [], [], []
        for ic in range(nsp):
            ypt.append(d[off:off + npty[ic]].copy())
            off += npty[ic]
        for ic in range(nsp):
            zpt.append(d[off:off + nptz[ic]].copy())
            off += nptz[ic]
        for ic in range(nsp):
            n = npty[ic] * nptz[ic]
            wghyz.append(d[off:off + n].reshape((npty[ic], nptz[ic]), order="F").copy())
            off += n
    return DumpState(it=it, t=float(rdata[0]), ndim=ndim, nx=nx2 - 2, fields=fields, species=species, nptx=nptx,
                     sptx_max=sptx_max, x0=float(rdata[8]), xlapse=float(rdata[9]), j0_norm=float(rdata[1]),
                     ompe=float(rdata[2]), targ_in=float(rdata[3]), targ_end=float(rdata[4]), lp_in=float(rdata[5]),
                     xp0_out=float(rdata[6]), xp1_out=float(rdata[7]), xpt=xpt, wghpt=wghpt, ypt=ypt, zpt=zpt,
                     wghyz=wghyz)


# ---- state holders (PicDevice, Oracle) --------------------------------------
def capture(holder, params0, it: int, t: float, sources=()) -> DumpState:
    """The dump of a simulation state holder (``aladyn_b200.sim.PicDevice`` or
    the oracle) whose run started from ``params0``; (it, t) are those of the
    next step; ``sources`` are the lattice plasma sources by species (None
    for species without one), from which the target extent, the xpt / wghpt
    table and the transverse lattice are written."""
    from .lattice import LatticeHost
    p = params0
    nsp = p.nsp
    xlapse, nptx, sptx_max, xmn = holder.window_state()
    species = [holder.get_species(ic) for ic in range(nsp)]
    srcs = list(sources) + [None] * (nsp - len(sources))
    hosts = [LatticeHost(p, s) if s is not None else None for s in srcs[:nsp]]
    targ_in = min((s.x_start for s in srcs[:nsp] if s is not None), default=0.0)
    targ_end = max((s.x_end for s in srcs[:nsp] if s is not None), default=0.0)
    x0 = xmn - p.xmn
    xpt = wghpt = None
    if targ_end > p.xmax + x0:
        nptx_max = max(h.sptx_max for h in hosts if h is not None)
        if nptx_max > XPT_MAX_COLUMNS:
            raise ValueError(f"a target of {nptx_max} lattice columns: the reference's xpt table of a dump "
                             f"holds at most {XPT_MAX_COLUMNS} here; give the plasma source a finite x_end")
        xpt = np.zeros((nptx_max, nsp))
        wghpt = np.zeros((nptx_max, nsp))
        for ic, h in enumerate(hosts):
            if h is None:
                continue
            j = np.arange(1, h.sptx_max + 1, dtype=np.float64)
            xpt[:h.sptx_max, ic] = h.s.x_start + (j - 0.5) * h.dxl
            wghpt[:h.sptx_max, ic] = float(h.s.wgh)
    ypt, zpt, wghyz = [], [], []
    for h in hosts:
        if h is None:
            ypt.append(np.zeros(0))
            zpt.append(np.zeros(0))
            wghyz.append(np.zeros((0, 0)))
            continue
        # the transverse lattice rows of this holder's box (loc_ypt: a block
        # of a y / z split keeps the rows inside its own bounds)
        yr = h.s.y_min + (np.arange(1, h.npty + 1) - 0.5) * h.dyl
        yr = yr[(yr > p.gymin) & (yr <= p.gymax)]
        if p.ndim == 3:
            zr = h.s.z_min + (np.arange(1, h.nptz + 1) - 0.5) * h.dzl
            zr = zr[(zr > p.gzmin) & (zr <= p.gzmax)]
        else:
            zr = np.zeros(1)
        ypt.append(yr)
        zpt.append(zr)
        wghyz.append(np.ones((len(yr), len(zr))))
    return DumpState(it=it, t=t, ndim=p.ndim, nx=p.nx, fields=holder.get_fields(), species=species,
                     nptx=[int(v) for v in nptx[:nsp]], sptx_max=[int(v) for v in sptx_max[:nsp]], x0=x0,
                     xlapse=xlapse, ompe=p.ompe, targ_in=targ_in, targ_end=targ_end, xpt=xpt, wghpt=wghpt,
                     ypt=ypt, zpt=zpt, wghyz=wghyz)


def shifted_params(params0, x0: float):
    """The run's parameters with the box moved by x0 along x, as restart moves
    x, xmin, xmax and the grid bounds (pic_dump.f90:515-526)."""
    p = type(params0).from_buffer_copy(params0)
    if x0 != 0.0:
        p.xmn += x0
        p.gxmin += x0
        p.gxmax += x0
        p.xmax += x0
    return p


def restore(holder, st: DumpState) -> None:
    """Fields, particles and window state of ``st`` into a holder created
    with ``shifted_params`` (plasma sources set beforehand)."""
    holder.set_fields(np.asfortranarray(st.fields))
    for ic, s in enumerate(st.species):
        if s.shape[0] > 0:
            holder.set_species(ic, np.asfortranarray(s))
    holder.set_window_state(st.xlapse, list(st.nptx) + [0] * (4 - len(st.nptx)))


# ---- several ranks: blocks of a y / z split ------------------------------------
def _block_files(dirpath: str, stem: str, rz: int) -> str:
    return os.path.join(dirpath, f"{stem}{rz:02d}.bin")


def write_dump_blocks(dirpath: str, states, layout, xmax: float) -> None:
    """Write the dumps of the blocks of a y / z split (``states[r]`` of block
    r = ry + npe_y * rz, the reference's mype order) as ``dump_data`` writes
    them with npe ranks (pic_dump.f90:84-377): ``Comm-data.bin`` from rank 0
    with ``npt_arr(1:npe, 1:nsp)``, ``dist_npy(1:npe_y, 1:nsp)`` and
    ``dist_npz(1:npe_z, 1:nsp)``; one ``EB-fieldsNN.bin`` and one
    ``ParticlesNN.bin`` per z column NN, the column's ranks one after the
    other in y order (each rank's whole local ebf, ghosts included, and its
    species' records); ``Dist-wgyz.bin`` with every rank's transverse lattice
    in mype order.  The reference places rank imody's fields at imody times
    its own length, so the y rows (and z planes) must split evenly."""
    ny_s, nz_s = layout.ny_s, layout.nz_s
    npe = ny_s * nz_s
    if len(states) != npe:
        raise ValueError(f"{len(states)} states for {npe} blocks")
    if len(set(layout.rows)) != 1 or len(set(layout.planes)) != 1:
        raise ValueError("a dump of several ranks needs rows and planes split evenly (ny_loc = ny/npe_y)")
    os.makedirs(dirpath, exist_ok=True)
    st0 = states[0]
    nsp = st0.nsp
    n1p, n2p, n3p = st0.fields.shape[:3]
    nd2 = 2 * st0.ndim
    with_xpt = st0.targ_end > xmax
    nptx_max = 0 if st0.xpt is None else st0.xpt.shape[0]
    if with_xpt and st0.xpt is None:
        raise ValueError("targ_end > xmax: the dump needs the xpt / wghpt table")
    rdata = np.array([st0.t, st0.j0_norm, st0.ompe, st0.targ_in, st0.targ_end, st0.lp_in, st0.xp0_out, st0.xp1_out,
                      st0.x0, st0.xlapse], dtype=np.float64)
    ndata = np.array([st0.it, n1p, n2p, n3p, nptx_max, st0.nx + 2, 0, nd2, 0, 0], dtype=np.int32)
    head = [rdata, ndata, np.asarray(st0.nptx, dtype=np.int32), np.asarray(st0.sptx_max, dtype=np.int32)]
    npt_arr = np.array([[st.species[ic].shape[0] for ic in range(nsp)] for st in states], dtype=np.int32)
    npty = np.array([[0 if st.ypt is None else len(st.ypt[ic]) for ic in range(nsp)] for st in states], dtype=np.int32)
    nptz = np.array([[0 if st.zpt is None else len(st.zpt[ic]) for ic in range(nsp)] for st in states], dtype=np.int32)
    dist_npy = np.array([npty[ry] for ry in range(ny_s)], dtype=np.int32)              # blocks (ry, 0)
    dist_npz = np.array([nptz[ny_s * rz] for rz in range(nz_s)], dtype=np.int32)     # blocks (0, rz)
    tail = [npt_arr.ravel(order="F"), dist_npy.ravel(order="F"), dist_npz.ravel(order="F")]
    path = os.path.join(dirpath, COMM)
    write_records(path, head)
    if with_xpt:
        blk = np.zeros(nsp * nptx_max, dtype=XPT_RECORD)
        blk["n0"] = 16
        blk["n1"] = 16
        blk["x"] = np.asarray(st0.xpt, dtype=np.float64).T.ravel()
        blk["w"] = np.asarray(st0.wghpt, dtype=np.float64).T.ravel()
        with open(path, "ab") as f:
            f.write(blk.tobytes())
    with open(path, "ab") as f:
        for r in tail:
            b = np.ascontiguousarray(r).tobytes()
            n = np.array([len(b)], dtype=np.int32).tobytes()
            f.write(n + b + n)
    with_part = int(npt_arr.sum()) > 0
    for rz in range(nz_s):
        with open(_block_files(dirpath, "EB-fields", rz), "wb") as f:
            for ry in range(ny_s):
                np.asfortranarray(states[ry + ny_s * rz].fields, dtype=np.float64).ravel(order="F").tofile(f)
        if with_part:
            with open(_block_files(dirpath, "Particles", rz), "wb") as f:
                for ry in range(ny_s):
                    for sp in states[ry + ny_s * rz].species:
                        if sp.shape[0] > 0:
                            np.asarray(sp, dtype=np.float64).ravel(order="F").tofile(f)
    if nsp > 0:
        with open(os.path.join(dirpath, DISTYZ), "wb") as f:
            for r, st in enumerate(states):
                for ic in range(nsp):
                    if npty[r, ic] > 0:
                        np.asarray(st.ypt[ic], dtype=np.float64).tofile(f)
                for ic in range(nsp):
                    if nptz[r, ic] > 0:
                        np.asarray(st.zpt[ic], dtype=np.float64).tofile(f)
                for ic in range(nsp):
                    if nptz[r, ic] > 0 and npty[r, ic] > 0:
                        np.asarray(st.wghyz[ic], dtype=np.float64).ravel(order="F").tofile(f)


def read_dump_blocks(dirpath: str, layout):
    """Read a dump of npe_y x npe_z ranks (``write_dump_blocks`` or the
    reference's ``dump_data``) into one DumpState per block, in mype order."""
    ny_s, nz_s = layout.ny_s, layout.nz_s
    npe = ny_s * nz_s
    path = os.path.join(dirpath, COMM)
    with open(path, "rb") as f:
        data = f.read()
    head, pos = _records_at(data, 0, 4, path)
    rdata = np.frombuffer(head[0], dtype=np.float64)
    ndata = np.frombuffer(head[1], dtype=np.int32)
    nptx = np.frombuffer(head[2], dtype=np.int32).astype(int).tolist()
    sptx_max = np.frombuffer(head[3], dtype=np.int32).astype(int).tolist()
    nsp = len(nptx)
    it, n1p, n2p, n3p, nptx_max, nx2, _, nd2 = (int(v) for v in ndata[:8])
    ndim = nd2 // 2
    tail_bytes = (8 + 4 * npe * nsp) + (8 + 4 * ny_s * nsp) + (8 + 4 * nz_s * nsp)
    xpt = wghpt = None
    nblk = len(data) - pos - tail_bytes
    if nblk > 0:
        if nblk != nsp * nptx_max * XPT_RECORD.itemsize:
            raise ValueError(f"{path}: {nblk} bytes of xpt records, expected {nsp * nptx_max} records")
        blk = np.frombuffer(data, dtype=XPT_RECORD, count=nsp * nptx_max, offset=pos)
        xpt = np.ascontiguousarray(blk["x"].reshape(nsp, nptx_max).T)
        wghpt = np.ascontiguousarray(blk["w"].reshape(nsp, nptx_max).T)
        pos += nblk
    recs, pos = _records_at(data, pos, 3, path)
    if pos != len(data):
        raise ValueError(f"{path}: {len(data) - pos} bytes after the last record")
    npt_arr = np.frombuffer(recs[0], dtype=np.int32).reshape((npe, nsp), order="F").astype(int)
    dist_npy = np.frombuffer(recs[1], dtype=np.int32).reshape((ny_s, nsp), order="F").astype(int)
    dist_npz = np.frombuffer(recs[2], dtype=np.int32).reshape((nz_s, nsp), order="F").astype(int)
    ndv = nd2 + 1
    ncell = n1p * n2p * n3p
    fields, species = [None] * npe, [None] * npe
    for rz in range(nz_s):
        raw = np.fromfile(_block_files(dirpath, "EB-fields", rz), dtype=np.float64)
        if raw.size % (ny_s * ncell):
            raise ValueError(f"EB-fields{rz:02d}.bin: {raw.size} values for {ny_s} ranks of {ncell} cells")
        nf = raw.size // (ny_s * ncell)
        for ry in range(ny_s):
            r = ry + ny_s * rz
            fields[r] = raw[ry * ncell * nf:(ry + 1) * ncell * nf].reshape((n1p, n2p, n3p, nf), order="F").copy(
                order="F")
        ppath = _block_files(dirpath, "Particles", rz)
        praw = np.fromfile(ppath, dtype=np.float64) if os.path.exists(ppath) else np.zeros(0)
        off = 0
        for ry in range(ny_s):
            r = ry + ny_s * rz
            species[r] = []
            for ic in range(nsp):
                n = int(npt_arr[r, ic])
                species[r].append(praw[off:off + n * ndv].reshape((n, ndv), order="F").copy(order="F"))
                off += n * ndv
        if off != praw.size:
            raise ValueError(f"Particles{rz:02d}.bin: {praw.size} values, expected {off}")
    lat = [(None, None, None)] * npe
    dpath = os.path.join(dirpath, DISTYZ)
    if os.path.exists(dpath):
        d = np.fromfile(dpath, dtype=np.float64)
        off = 0
        lat = []
        for r in range(npe):
            ry, rz = r % ny_s, r // ny_s
            ny_r, nz_r = dist_npy[ry], dist_npz[rz]
            ypt, zpt, wghyz = [], [], []
            for ic in range(nsp):
                ypt.append(d[off:off + ny_r[ic]].copy())
                off += ny_r[ic]
            for ic in range(nsp):
                zpt.append(d[off:off + nz_r[ic]].copy())
                off += nz_r[ic]
            for ic in range(nsp):
                n = ny_r[ic] * nz_r[ic] if (ny_r[ic] > 0 and nz_r[ic] > 0) else 0
                wghyz.append(d[off:off + n].reshape((ny_r[ic], nz_r[ic]), order="F").copy())
                off += n
            lat.append((ypt, zpt, wghyz))
        if off != d.size:
            raise ValueError(f"{DISTYZ}: {d.size} values, expected {off}")
    out = []
    for r in range(npe):
        out.append(DumpState(it=it, t=float(rdata[0]), ndim=ndim, nx=nx2 - 2, fields=fields[r], species=species[r],
                             nptx=list(nptx), sptx_max=list(sptx_max), x0=float(rdata[8]), xlapse=float(rdata[9]),
                             j0_norm=float(rdata[1]), ompe=float(rdata[2]), targ_in=float(rdata[3]),
                             targ_end=float(rdata[4]), lp_in=float(rdata[5]), xp0_out=float(rdata[6]),
                             xp1_out=float(rdata[7]), xpt=xpt, wghpt=wghpt, ypt=lat[r][0], zpt=lat[r][1],
                             wghyz=lat[r][2]))
    return out
