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

LOW, HIGH = 0, 1


# ---- layout -------------------------------------------------------------------
class SlabLayout:
    """Rows of a global box split into ``nslabs`` slabs along y: slab r owns
    the global interior rows j0 .. j0 + rows - 1 (0-based), the first
    ``ny % nslabs`` slabs one row more (the loc_ygrid split)."""

    def __init__(self, params: AgpuParams, nslabs: int):
        if params.ndim < 2:
            raise ValueError("a y decomposition needs ndim >= 2")
        if nslabs < 1 or params.ny < 3 * nslabs:
            raise ValueError(f"{params.ny} rows cannot be split into {nslabs} slabs of at least 3 rows")
        self.p = params
        self.n = nslabs
        base, extra = divmod(params.ny, nslabs)
        self.rows = [base + (1 if r < extra else 0) for r in range(nslabs)]
        self.j0 = [sum(self.rows[:r]) for r in range(nslabs)]

    def y_at(self, j0: int) -> float:
        """y of the slab boundary before global row j0 (the box's own
        bounds at both ends)."""
        if j0 == 0:
            return self.p.gymin
        if j0 == self.p.ny:
            return self.p.gymax
        return self.p.ymn + self.p.dy * j0

    def params(self, r: int, capacity=None) -> AgpuParams:
        """The params of slab r: ny = its rows, ymn = gymin = y of its first
        row, gymax = y after its last row; everything else global."""
        q = AgpuParams()
        C.memmove(C.byref(q), C.byref(self.p), C.sizeof(AgpuParams))
        q.ny = self.rows[r]
        lo, hi = self.y_at(self.j0[r]), self.y_at(self.j0[r] + self.rows[r])
        q.ymn = self.p.ymn if r == 0 else lo
        q.gymin, q.gymax = lo, hi
        if capacity is not None:
            for i in range(4):
                q.capacity[i] = int(capacity[i])
        return q

    def shared(self, r: int):
        """(low side shared, high side shared) of slab r."""
        return r > 0, r < self.n - 1

    def assemble(self, arrays):
        """One (n1p, n2p, n3p, nc) array of the global box from the slabs'
        arrays: each slab's interior rows, the low ghost rows of slab 0 and
        the high ghost rows of the last slab."""
        import numpy as np
        first = arrays[0]
        n1p, _, n3p, nc = first.shape
        out = np.zeros((n1p, self.p.ny + 5, n3p, nc), order="F")
        out[:, 0:2] = first[:, 0:2]
        for r, a in enumerate(arrays):
            out[:, 2 + self.j0[r]:2 + self.j0[r] + self.rows[r]] = a[:, 2:2 + self.rows[r]]
        last = arrays[-1]
        out[:, self.p.ny + 2:] = last[:, self.rows[-1] + 2:]
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
    """Slab r of a layout on its PicDevice: registers the exchange hook and
    carries out the exchanges the library asks for."""

    def __init__(self, layout: SlabLayout, rank: int, dev, exchanger, emigrant_capacity: int = 1 << 16):
        import torch
        self.torch = torch
        self.layout = layout
        self.rank = rank
        self.dev = dev
        self.ex = exchanger
        self.lib = dev.lib
        self.lo, self.hi = layout.shared(rank)
        self.nbr = {}
        if self.lo:
            self.nbr[LOW] = rank - 1
        if self.hi:
            self.nbr[HIGH] = rank + 1
        p = layout.params(rank)
        self.nf, self.nc = p.nfield, p.curr_ndim
        self.jy1, self.jy2 = 3, p.ny + 2
        self.ndv = 7 if p.ndim == 3 else 5
        self.device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
        self.ecap = int(emigrant_capacity)
        self.error = None
        self.calls = {AGPU_HALO_FIELDS: 0, AGPU_HALO_PARTICLES: 0, AGPU_HALO_CURRENTS: 0, AGPU_HALO_E: 0,
                      AGPU_HALO_B: 0}
        self.migrated = 0
        self._fn = HALO_FN(self._hook)
        check(self.lib.agpu_set_subdomain(dev.h, int(self.lo), int(self.hi), self._fn, None), "agpu_set_subdomain")
        self._stream = torch.cuda.ExternalStream(dev.stream()) if torch.cuda.is_available() else None

    # -- helpers
    def _size(self, ncomp, nrows):
        n = C.c_int64()
        check(self.lib.agpu_halo_size(self.dev.h, ncomp, nrows, C.byref(n)), "agpu_halo_size")
        return n.value

    def _buf(self, n):
        return self.torch.empty(max(int(n), 1), dtype=self.torch.float64, device=self.device)

    def _pack(self, what, ic1, ic2, j1, nrows):
        b = self._buf(self._size(ic2 - ic1 + 1, nrows))
        check(self.lib.agpu_halo_pack(self.dev.h, what, ic1, ic2, j1, nrows, C.c_void_p(b.data_ptr())), "agpu_halo_pack")
        return b

    def _unpack(self, what, ic1, ic2, j1, nrows, buf, mode):
        ptr = C.c_void_p(buf.data_ptr()) if buf is not None else None
        check(self.lib.agpu_halo_unpack(self.dev.h, what, ic1, ic2, j1, nrows, ptr, mode), "agpu_halo_unpack")

    def _sync_for_peers(self):
        # the thread exchanger reads the buffers from the neighbours' streams
        if isinstance(self.ex, ThreadExchanger):
            self.dev.synchronize()

    def _rows(self, tag, what, ic1, ic2, down, up, add=False):
        """Send `down` rows from the bottom of my interior to the low
        neighbour (its high ghost rows) and `up` rows from the top to the
        high neighbour (its low ghost rows); with add, send my ghost rows
        instead (down: the 2 below jy1, up: the 3 above jy2) and add them
        into the neighbours' edge rows, then zero mine."""
        sends, sizes, place = {}, {}, {}
        if self.lo:
            n_send = down
            j_send = (self.jy1 - down) if add else self.jy1
            sends[self.nbr[LOW]] = self._pack(what, ic1, ic2, j_send, n_send)
            n_recv = up
            j_recv = self.jy1 if add else self.jy1 - up
            sizes[self.nbr[LOW]] = self._size(ic2 - ic1 + 1, n_recv)
            place[self.nbr[LOW]] = (j_recv, n_recv)
        if self.hi:
            n_send = up
            j_send = (self.jy2 + 1) if add else self.jy2 - up + 1
            sends[self.nbr[HIGH]] = self._pack(what, ic1, ic2, j_send, n_send)
            n_recv = down
            j_recv = (self.jy2 - down + 1) if add else self.jy2 + 1
            sizes[self.nbr[HIGH]] = self._size(ic2 - ic1 + 1, n_recv)
            place[self.nbr[HIGH]] = (j_recv, n_recv)
        self._sync_for_peers()
        got = self.ex.exchange(self.rank, tag, sends, sizes, self.device)
        for src, buf in got.items():
            j1, nr = place[src]
            self._unpack(what, ic1, ic2, j1, nr, buf, 1 if add else 0)
        if add:
            if self.lo:
                self._unpack(what, ic1, ic2, self.jy1 - down, down, None, 2)
            if self.hi:
                self._unpack(what, ic1, ic2, self.jy2 + 1, up, None, 2)
        self._sync_for_peers()
        self.ex.done(self.rank)

    def _particles(self, ic):
        torch = self.torch
        sends, counts = {}, {}
        for side, dst in self.nbr.items():
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
            # compact the ndv columns of leading dimension ecap to leading dimension k
            sends[dst] = buf.view(self.ndv, self.ecap)[:, :k].contiguous().view(-1)
            counts[dst] = k
        self._sync_for_peers()
        got_n = self.ex.exchange_counts(self.rank, ("n", ic), counts)
        sizes = {src: got_n[src] * self.ndv for src in got_n}
        got = self.ex.exchange(self.rank, ("p", ic), sends, sizes, self.device)
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
                    self._rows(("f",), 0, 1, self.nf, 2, 2)
                elif point == AGPU_HALO_E:
                    # fill_ebfield_yzxbdsdata(ef, 1, curr_ndim, str = 1, stl = 2)
                    self._rows(("e",), 0, 1, self.nc, 2, 1)
                elif point == AGPU_HALO_B:
                    # fill_ebfield_yzxbdsdata(ef, curr_ndim + 1, nfield, str = 2, stl = 1)
                    self._rows(("b",), 0, self.nc + 1, self.nf, 1, 2)
                elif point == AGPU_HALO_CURRENTS:
                    # fill_curr_yzxbdsdata: 2 ghost rows down, 3 up, summed
                    self._rows(("j",), 1, 1, self.nc, 2, 3, add=True)
                elif point == AGPU_HALO_PARTICLES:
                    self._particles(ic)
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


__all__ = ["SlabLayout", "Slab", "ThreadExchanger", "DistExchanger", "run_threads", "LOW", "HIGH"]
