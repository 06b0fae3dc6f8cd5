"""Domain decomposition of one simulation into slabs of rows along y.

The reference splits its box over MPI ranks in y and z
(src/parallel/parallel.F90:75-140) and exchanges, inside each step, the
field halos (fill_ebfield_yzxbdsdata, src/parallel/mpi_field_interface.f90:
361-658), the ghost currents (fill_curr_yzxbdsdata,
src/parallel/mpi_curr_interface.f90:51-159) and the particles that cross a
rank boundary (part_prl_exchange, src/parallel/mpi_part_interface.f90:
246-466).  Here one handle holds one slab (nprocy slabs, npe_z = 1); the
library calls the slab's hook at each exchange point of the step and the
hook moves packed rows and particle records between neighbours:

* ``DistExchanger``: one process per GPU, ``torch.distributed`` point-to-point
  sends and receives (NCCL over NVLink on GPUs, gloo on CPU tensors), queued
  on the handle's own CUDA stream so the packing kernels, the transfer and
  the unpacking stay ordered without a host wait;
* ``ThreadExchanger``: several slabs of one process (one host thread per
  slab, for instance on one GPU), each slab reading its neighbours' packed
  buffers directly; the host threads meet at a barrier after packing and
  after unpacking, so no kernel ever waits on another one.

Rows move whole (every x and z node, ghosts included), so a slab sees its
neighbour's boundary values exactly as one box would; the results differ
from one box only by the order of floating-point sums (ghost currents added
after the slab's own) and by each slab's local coordinates.
"""
from __future__ import annotations

import ctypes as C
import threading

from . import abi
from .abi import (AGPU_E_STATE, AGPU_HALO_B, AGPU_HALO_CURRENTS, AGPU_HALO_E, AGPU_HALO_FIELDS,
                  AGPU_HALO_PARTICLES, AgpuParams, HALO_FN, check)

LOW, HIGH, ZLOW, ZHIGH = 0, 1, 2, 3


def _split(n: int, parts: int):
    base, extra = divmod(n, parts)
    sizes = [base + (1 if r < extra else 0) for r in range(parts)]
    return sizes, [sum(sizes[:r]) for r in range(parts)]


# ---- layout -------------------------------------------------------------------
class SlabLayout:
    """A global box split into ``nslabs`` slabs of rows along y and, in 3D,
    ``nzslabs`` blocks of planes along z (the reference's nprocy x nprocz
    split): block r = ry + nslabs * rz owns the global interior rows
    j0[ry] .. j0[ry] + rows[ry] - 1 and planes k0[rz] .. k0[rz] + planes[rz]
    - 1 (0-based), the first ``ny % nslabs`` (``nz % nzslabs``) one more
    (the loc_ygrid / loc_zgrid split)."""

    def __init__(self, params: AgpuParams, nslabs: int, nzslabs: int = 1):
        if params.ndim < 2:
            raise ValueError("a y decomposition needs ndim >= 2")
        if nslabs < 1 or params.ny < 3 * nslabs:
            raise ValueError(f"{params.ny} rows cannot be split into {nslabs} slabs of at least 3 rows")
        if nzslabs < 1 or (nzslabs > 1 and (params.ndim < 3 or params.nz < 3 * nzslabs)):
            raise ValueError(f"the z planes cannot be split into {nzslabs} blocks of at least 3 planes")
        self.p = params
        self.ny_s, self.nz_s = nslabs, nzslabs
        self.n = nslabs * nzslabs
        self.rows, self.j0 = _split(params.ny, nslabs)
        nz = params.nz if params.ndim == 3 else 1
        self.planes, self.k0 = _split(nz, nzslabs)

    def coords(self, r: int):
        return r % self.ny_s, r // self.ny_s

    def y_at(self, j0: int) -> float:
        """y of the slab boundary before global row j0 (the box's own
        bounds at both ends)."""
        if j0 == 0:
            return self.p.gymin
        if j0 == self.p.ny:
            return self.p.gymax
        return self.p.ymn + self.p.dy * j0

    def z_at(self, k0: int) -> float:
        if k0 == 0:
            return self.p.gzmin
        if k0 == self.p.nz:
            return self.p.gzmax
        return self.p.zmn + self.p.dz * k0

    def params(self, r: int, capacity=None) -> AgpuParams:
        """The params of block r: ny (nz) = its rows (planes), ymn = gymin
        = y of its first row, gymax = y after its last row, z alike;
        everything else global."""
        ry, rz = self.coords(r)
        q = AgpuParams()
        C.memmove(C.byref(q), C.byref(self.p), C.sizeof(AgpuParams))
        q.ny = self.rows[ry]
        lo, hi = self.y_at(self.j0[ry]), self.y_at(self.j0[ry] + self.rows[ry])
        q.ymn = self.p.ymn if ry == 0 else lo
        q.gymin, q.gymax = lo, hi
        if self.nz_s > 1:
            q.nz = self.planes[rz]
            lo, hi = self.z_at(self.k0[rz]), self.z_at(self.k0[rz] + self.planes[rz])
            q.zmn = self.p.zmn if rz == 0 else lo
            q.gzmin, q.gzmax = lo, hi
        if capacity is not None:
            for i in range(4):
                q.capacity[i] = int(capacity[i])
        return q

    def shared(self, r: int):
        """(low y, high y, low z, high z) side shared, of block r."""
        ry, rz = self.coords(r)
        return ry > 0, ry < self.ny_s - 1, rz > 0, rz < self.nz_s - 1

    def neighbours(self, r: int) -> dict:
        lo, hi, zlo, zhi = self.shared(r)
        out = {}
        if lo:
            out[LOW] = r - 1
        if hi:
            out[HIGH] = r + 1
        if zlo:
            out[ZLOW] = r - self.ny_s
        if zhi:
            out[ZHIGH] = r + self.ny_s
        return out

    def local(self, r: int, a):
        """Block r's part of a global (n1p, n2p, n3p, nc) array, ghosts
        included (what the block's own handle holds)."""
        import numpy as np
        ry, rz = self.coords(r)
        j0, nr = self.j0[ry], self.rows[ry]
        if self.nz_s == 1:
            return np.asfortranarray(a[:, j0:j0 + nr + 5])
        k0, nk = self.k0[rz], self.planes[rz]
        return np.asfortranarray(a[:, j0:j0 + nr + 5, k0:k0 + nk + 5])

    def assemble(self, arrays):
        """One (n1p, n2p, n3p, nc) array of the global box from the blocks'
        arrays: each block's interior, and the ghost rows (planes) of the
        blocks at the box's sides."""
        import numpy as np
        first = arrays[0]
        n1p, _, n3p_loc, nc = first.shape
        n3p = (self.p.nz + 5) if self.p.ndim == 3 else 1
        out = np.zeros((n1p, self.p.ny + 5, n3p, nc), order="F")
        for r, a in enumerate(arrays):
            ry, rz = self.coords(r)
            j0, nr = self.j0[ry], self.rows[ry]
            jl = 0 if ry == 0 else 2
            jh = nr + 5 if ry == self.ny_s - 1 else nr + 2
            if self.nz_s == 1:
                out[:, j0 + jl:j0 + jh] = a[:, jl:jh]
                continue
            k0, nk = self.k0[rz], self.planes[rz]
            kl = 0 if rz == 0 else 2
            kh = nk + 5 if rz == self.nz_s - 1 else nk + 2
            out[:, j0 + jl:j0 + jh, k0 + kl:k0 + kh] = a[:, jl:jh, kl:kh]
        return out


# ---- exchangers -----------------------------------------------------------------
class ThreadExchanger:
    """Neighbour exchange between slabs that live in one process, one host
    thread per slab.  ``exchange`` publishes this slab's send buffers, waits
    for every slab to do the same, and returns the neighbours' buffers for
    this slab; ``done`` is the second meeting point, after which a slab may
    overwrite its send buffers again."""

    def __init__(self, nslabs: int, timeout: float = 120.0):
        self.n = nslabs
        self.box = {}
        self.lock = threading.Lock()
        self.barrier = threading.Barrier(nslabs, timeout=timeout)

    def exchange(self, rank: int, tag, sends: dict, recv_sizes: dict, device):
        with self.lock:
            for dst, t in sends.items():
                self.box[(tag, rank, dst)] = t
        self.barrier.wait()
        with self.lock:
            got = {src: self.box[(tag, src, rank)] for src in recv_sizes}
        return got

    def exchange_counts(self, rank: int, tag, counts: dict):
        with self.lock:
            for dst, c in counts.items():
                self.box[(tag, rank, dst)] = int(c)
        self.barrier.wait()
        with self.lock:
            return {src: self.box[(tag, src, rank)] for src in counts}

    def done(self, rank: int):
        self.barrier.wait()
        with self.lock:
            for key in [k for k in self.box if k[1] == rank]:
                del self.box[key]
        self.barrier.wait()


class DistExchanger:
    """Neighbour exchange over ``torch.distributed`` point-to-point calls
    (one slab per rank of the group, rank r = slab r)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def exchange(self, rank: int, tag, sends: dict, recv_sizes: dict, device):
        import torch
        dist = self.dist
        recvs = {src: torch.empty(int(n), dtype=torch.float64, device=device) for src, n in recv_sizes.items()}
        ops = []
        # empty blocks (no particles crossed) are not sent: both sides know
        # the sizes beforehand
        for src, t in recvs.items():
            if t.numel() > 0:
                ops.append(dist.P2POp(dist.irecv, t, src, group=self.group))
        for dst, t in sends.items():
            if t.numel() > 0:
                ops.append(dist.P2POp(dist.isend, t, dst, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        return recvs

    def exchange_counts(self, rank: int, tag, counts: dict):
        import torch
        dist = self.dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        send = {d: torch.tensor([int(c)], dtype=torch.int64, device=dev) for d, c in counts.items()}
        recv = {s: torch.zeros(1, dtype=torch.int64, device=dev) for s in counts}
        ops = [dist.P2POp(dist.irecv, t, s, group=self.group) for s, t in recv.items()]
        ops += [dist.P2POp(dist.isend, t, d, group=self.group) for d, t in send.items()]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        return {s: int(t.item()) for s, t in recv.items()}

    def done(self, rank: int):
        pass


# ---- one slab ----------------------------------------------------------------
class Slab:
    """Block r of a layout on its PicDevice: registers the exchange hook and
    carries out the exchanges the library asks for (the y rows first, then,
    with a z split, the z planes over the whole y range, ghosts included)."""

    def __init__(self, layout: SlabLayout, rank: int, dev, exchanger, emigrant_capacity: int = 1 << 16):
        import torch
        self.torch = torch
        self.layout = layout
        self.rank = rank
        self.dev = dev
        self.ex = exchanger
        self.lib = dev.lib
        self.lo, self.hi, self.zlo, self.zhi = layout.shared(rank)
        self.nbr = layout.neighbours(rank)
        self.zsplit = layout.nz_s > 1
        p = layout.params(rank)
        self.nf, self.nc = p.nfield, p.curr_ndim
        self.jy1, self.jy2 = 3, p.ny + 2
        self.kz1, self.kz2 = 3, (p.nz + 2 if p.ndim == 3 else 1)
        self.ndv = 7 if p.ndim == 3 else 5
        self.device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
        self.ecap = int(emigrant_capacity)
        self.error = None
        self.calls = {AGPU_HALO_FIELDS: 0, AGPU_HALO_PARTICLES: 0, AGPU_HALO_CURRENTS: 0, AGPU_HALO_E: 0,
                      AGPU_HALO_B: 0}
        self.migrated = 0
        self._fn = HALO_FN(self._hook)
        if self.zsplit:
            shared = (C.c_int32 * 4)(int(self.lo), int(self.hi), int(self.zlo), int(self.zhi))
            check(self.lib.agpu_set_subdomain_yz(dev.h, shared, self._fn, None), "agpu_set_subdomain_yz")
        else:
            check(self.lib.agpu_set_subdomain(dev.h, int(self.lo), int(self.hi), self._fn, None), "agpu_set_subdomain")
        self._stream = torch.cuda.ExternalStream(dev.stream()) if torch.cuda.is_available() else None

    # -- helpers
    def _size(self, axis, ncomp, n):
        out = C.c_int64()
        f = self.lib.agpu_halo_size if axis == "y" else self.lib.agpu_halo_size_z
        check(f(self.dev.h, ncomp, n, C.byref(out)), "agpu_halo_size")
        return out.value

    def _buf(self, n):
        return self.torch.empty(max(int(n), 1), dtype=self.torch.float64, device=self.device)

    def _pack(self, axis, what, ic1, ic2, first, n):
        b = self._buf(self._size(axis, ic2 - ic1 + 1, n))
        f = self.lib.agpu_halo_pack if axis == "y" else self.lib.agpu_halo_pack_z
        check(f(self.dev.h, what, ic1, ic2, first, n, C.c_void_p(b.data_ptr())), "agpu_halo_pack")
        return b

    def _unpack(self, axis, what, ic1, ic2, first, n, buf, mode):
        ptr = C.c_void_p(buf.data_ptr()) if buf is not None else None
        f = self.lib.agpu_halo_unpack if axis == "y" else self.lib.agpu_halo_unpack_z
        check(f(self.dev.h, what, ic1, ic2, first, n, ptr, mode), "agpu_halo_unpack")

    def _sync_for_peers(self):
        # the thread exchanger reads the buffers from the neighbours' streams
        if isinstance(self.ex, ThreadExchanger):
            self.dev.synchronize()

    def _layers(self, axis, tag, what, ic1, ic2, down, up, add=False):
        """Along y (rows) or z (planes): send `down` layers from the bottom
        of my interior to the low neighbour (its high ghost layers) and `up`
        layers from the top to the high neighbour (its low ghost layers);
        with add, send my ghost layers instead (down: the 2 below the
        interior, up: the 3 above) and add them into the neighbours' edge
        layers, then zero mine."""
        lo_side, hi_side = (LOW, HIGH) if axis == "y" else (ZLOW, ZHIGH)
        i1, i2 = (self.jy1, self.jy2) if axis == "y" else (self.kz1, self.kz2)
        sends, sizes, place = {}, {}, {}
        nc = ic2 - ic1 + 1
        if lo_side in self.nbr:
            src = self.nbr[lo_side]
            sends[src] = self._pack(axis, what, ic1, ic2, (i1 - down) if add else i1, down)
            sizes[src] = self._size(axis, nc, up)
            place[src] = (i1 if add else i1 - up, up)
        if hi_side in self.nbr:
            src = self.nbr[hi_side]
            sends[src] = self._pack(axis, what, ic1, ic2, (i2 + 1) if add else i2 - up + 1, up)
            sizes[src] = self._size(axis, nc, down)
            place[src] = ((i2 - down + 1) if add else i2 + 1, down)
        self._sync_for_peers()
        got = self.ex.exchange(self.rank, tag + (axis,), sends, sizes, self.device)
        for src, buf in got.items():
            first, n = place[src]
            self._unpack(axis, what, ic1, ic2, first, n, buf, 1 if add else 0)
        if add:
            if lo_side in self.nbr:
                self._unpack(axis, what, ic1, ic2, i1 - down, down, None, 2)
            if hi_side in self.nbr:
                self._unpack(axis, what, ic1, ic2, i2 + 1, up, None, 2)
        self._sync_for_peers()
        self.ex.done(self.rank)

    def _exchange(self, tag, what, ic1, ic2, down, up, add=False):
        self._layers("y", tag, what, ic1, ic2, down, up, add)
        if self.zsplit:
            self._layers("z", tag, what, ic1, ic2, down, up, add)

    def _particles(self, ic, sides):
        sends, counts = {}, {}
        for side in sides:
            if side not in self.nbr:
                continue
            dst = self.nbr[side]
            while True:
                buf = self._buf(self.ecap * self.ndv)
                n = C.c_int64()
                rc = self.lib.agpu_halo_emigrants(self.dev.h, ic, side, C.c_void_p(buf.data_ptr()), self.ecap,
                                                  C.byref(n))
                if rc == abi.AGPU_E_CAPACITY:
                    self.ecap = max(2 * self.ecap, int(n.value) + 1)
                    continue
                check(rc, "agpu_halo_emigrants")
                break
            k = int(n.value)
            # the ndv columns of leading dimension ecap to leading dimension k
            sends[dst] = buf.view(self.ndv, self.ecap)[:, :k].contiguous().view(-1)
            counts[dst] = k
        self._sync_for_peers()
        got_n = self.ex.exchange_counts(self.rank, ("n", ic, sides[0]), counts)
        sizes = {src: got_n[src] * self.ndv for src in got_n}
        got = self.ex.exchange(self.rank, ("p", ic, sides[0]), sends, sizes, self.device)
        for src in sorted(got):
            n = got_n[src]
            if n > 0:
                check(self.lib.agpu_halo_immigrants(self.dev.h, ic, C.c_void_p(got[src].data_ptr()), n, n),
                      "agpu_halo_immigrants")
                self.migrated += n
        self._sync_for_peers()
        self.ex.done(self.rank)

    # -- the hook the library calls inside agpu_step
    def _hook(self, user, h, point, ic):
        try:
            self.calls[point] += 1
            ctx = self.torch.cuda.stream(self._stream) if self._stream is not None else _Null()
            with ctx:
                if point == AGPU_HALO_FIELDS:
                    self._exchange(("f",), 0, 1, self.nf, 2, 2)
                elif point == AGPU_HALO_E:
                    # fill_ebfield_yzxbdsdata(ef, 1, curr_ndim, str = 1, stl = 2)
                    self._exchange(("e",), 0, 1, self.nc, 2, 1)
                elif point == AGPU_HALO_B:
                    # fill_ebfield_yzxbdsdata(ef, curr_ndim + 1, nfield, str = 2, stl = 1)
                    self._exchange(("b",), 0, self.nc + 1, self.nf, 1, 2)
                elif point == AGPU_HALO_CURRENTS:
                    # fill_curr_yzxbdsdata: 2 ghost layers down, 3 up, summed
                    self._exchange(("j",), 1, 1, self.nc, 2, 3, add=True)
                elif point == AGPU_HALO_PARTICLES:
                    # part_prl_exchange: through the y sides, then the z sides
                    self._particles(ic, (LOW, HIGH))
                    if self.zsplit:
                        self._particles(ic, (ZLOW, ZHIGH))
            return 0
        except Exception as e:  # reported by the step's return code
            self.error = e
            return AGPU_E_STATE


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def run_threads(slabs, fn):
    """Run fn(slab) for every slab, one host thread each; re-raise the first
    failure (a slab hook's own error first)."""
    errors = [None] * len(slabs)

    def work(i):
        import torch
        if torch.cuda.is_available():
            torch.cuda.set_device(slabs[i].device)
        try:
            fn(slabs[i])
        except Exception as e:
            errors[i] = e
            if isinstance(slabs[i].ex, ThreadExchanger):
                slabs[i].ex.barrier.abort()

    ths = [threading.Thread(target=work, args=(i,)) for i in range(len(slabs))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for s in slabs:
        if s.error is not None:
            raise s.error
    for e in errors:
        if e is not None:
            raise e


__all__ = ["SlabLayout", "Slab", "ThreadExchanger", "DistExchanger", "run_threads", "LOW", "HIGH", "ZLOW", "ZHIGH"]
