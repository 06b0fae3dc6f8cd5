"""Host-side lattice plasma columns, as the reference's host injects them.

In the reference the moving-window injection runs on the host:
``particles_inject`` picks the lattice columns that entered the box
(src/dynamics/window.f90:106-184) and ``add_particles`` writes their records
(window.f90:39-104).  ``LatticeHost`` restates that for the library's jittered
lattice (same Philox4x32-10 counters and the same FP64 expressions as the
device kernel, so the records are bit-identical), producing Fortran-layout
records a host passes to ``agpu_window_inject``.
"""
from __future__ import annotations

import math

import numpy as np

from .sim import pack_slot

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = np.uint32(0x9E3779B9)
_W1 = np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0: int, k1: int):
    """Vectorised Philox4x32-10 (Salmon et al., SC'11) on uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint32).copy()
    c1 = np.asarray(c1, dtype=np.uint32).copy()
    c2 = np.asarray(c2, dtype=np.uint32).copy()
    c3 = np.asarray(c3, dtype=np.uint32).copy()
    k0 = np.uint32(k0 & 0xFFFFFFFF)
    k1 = np.uint32(k1 & 0xFFFFFFFF)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _M0 * c0.astype(np.uint64)
            p1 = _M1 * c2.astype(np.uint64)
            hi0 = (p0 >> np.uint64(32)).astype(np.uint32)
            lo0 = (p0 & _MASK).astype(np.uint32)
            hi1 = (p1 >> np.uint64(32)).astype(np.uint32)
            lo1 = (p1 & _MASK).astype(np.uint32)
            n0 = hi1 ^ c1 ^ k0
            n2 = hi0 ^ c3 ^ k1
            c0, c1, c2, c3 = n0, lo1, n2, lo0
            k0 = np.uint32((int(k0) + int(_W0)) & 0xFFFFFFFF)
            k1 = np.uint32((int(k1) + int(_W1)) & 0xFFFFFFFF)
    return c0, c1, c2, c3


class LatticeHost:
    """Column bookkeeping and records of one lattice plasma source."""

    def __init__(self, params, src):
        self.p = params
        self.s = src
        self.dxl = params.dx / float(src.npx)
        self.dyl = params.dy / float(src.npy)
        self.dzl = params.dz / float(src.npz)
        self.sptx_max = int(math.floor((src.x_end - src.x_start) / self.dxl + 1e-9))
        self.npty = int(math.floor((src.y_max - src.y_min) / self.dyl + 1e-9))
        self.nptz = int(math.floor((src.z_max - src.z_min) / self.dzl + 1e-9)) if params.ndim == 3 else 1
        self.nptx = 0

    def xpt(self, ix):
        return self.s.x_start + (float(ix) - 0.5) * self.dxl

    def columns_end(self, i1: int, xmx: float, reference_quirk: bool) -> int:
        """particles_inject's search (window.f90:124-136)."""
        if i1 > self.sptx_max:
            return i1 - 1
        ix = i1
        while ix <= self.sptx_max:
            if self.xpt(ix) > xmx:
                break
            ix += 1
        i2 = ix - 1
        if reference_quirk and ix == self.sptx_max:
            i2 = ix
        return i2

    def records(self, i1: int, i2: int) -> np.ndarray:
        """add_particles order (k, j, ix with x fastest) for columns i1..i2."""
        p, s = self.p, self.s
        ncol = i2 - i1 + 1
        if ncol <= 0:
            return np.zeros((0, 7 if p.ndim == 3 else 5), order="F")
        q = np.arange(ncol * self.npty * self.nptz, dtype=np.int64)
        ix = i1 + q % ncol
        j = 1 + (q // ncol) % self.npty
        k = 1 + q // (ncol * self.npty)
        r0, r1, r2, _ = philox4x32_10(ix.astype(np.uint32), j.astype(np.uint32), k.astype(np.uint32),
                                      np.full(q.shape, s.ic, dtype=np.uint32), s.seed & 0xFFFFFFFF, s.seed >> 32)
        u = 1.0 / 4294967296.0
        jx = s.jitter * (r0.astype(np.float64) * u - 0.5)
        jy = s.jitter * (r1.astype(np.float64) * u - 0.5)
        jz = s.jitter * (r2.astype(np.float64) * u - 0.5)
        x = s.x_start + ((ix.astype(np.float64) - 0.5) + jx) * self.dxl
        y = s.y_min + ((j.astype(np.float64) - 0.5) + jy) * self.dyl
        slot = pack_slot(s.charge, s.part_ind, np.float32(s.wgh))
        if p.ndim == 3:
            z = s.z_min + ((k.astype(np.float64) - 0.5) + jz) * self.dzl
            rec = np.zeros((q.size, 7), order="F")
            rec[:, 0], rec[:, 1], rec[:, 2] = x, y, z
            rec[:, 6] = slot
        else:
            rec = np.zeros((q.size, 5), order="F")
            rec[:, 0], rec[:, 1] = x, y
            rec[:, 4] = slot
        return rec

    def inject_after_shift(self, xmax: float) -> np.ndarray:
        """Records a host injects after a window shift to grid end xmax."""
        if not (self.s.x_start <= xmax < self.s.x_end):
            return self.records(1, 0)
        i1 = 1 + self.nptx
        i2 = self.columns_end(i1, xmax, True)
        self.nptx = i2
        if i2 > i1:
            return self.records(i1, i2)
        return self.records(1, 0)
