"""Discrete continuity residual of one step, computed on the host in FP64.

The Esirkepov deposit (src/particles/grid_part_connect.f90:956-1334) is
built so that the current of a step satisfies the discrete continuity
equation exactly for the charge density of the qden shapes
(src/particles/grid_part_lib.f90:337-358, 388-417):

    rho1(n) - rho0(n) + c * sum_a (J_a(n) - J_a(n - e_a)) = 0,

with rho0 / rho1 the densities of the particles before / after the step,
J the raw deposited current (before the djc normalisation) and c = 1/2 in
2D, 1/3 in 3D (djc = dx/2 or dx/3, src/start/set_init_param.f90:92-103).
``step_residual`` evaluates the left-hand side from the particle records
(absolute positions, packed charge and weight) and the currents that
``agpu_get_currents`` returns (djc times the raw sums), so the same check
runs on either precision form of the device and on the oracle.  The weight
of each particle is real(charge * wgh, sp), as the deposit rounds it.

The fold of the ghost currents into the boundary cells (jc_xyzbd) and the
removal of particles at the box edges break the identity near the edges, so
callers keep the particles away from them or pass ``margin``.
"""
from __future__ import annotations

import numpy as np

from .sim import unpack_slot

SHX = 3.0  # the sp constant shx of grid_part_lib.f90:32


def _qden(xl: np.ndarray):
    """Quadratic weights on the three integer nodes i-1, i, i+1 (1-based i)
    of local grid coordinates xl (qden_*_wgh)."""
    xx = SHX + xl
    i = np.floor(xx + 0.5).astype(np.int64)
    s = xx - i
    s2 = s * s
    a1 = 0.75 - s2
    a2 = 0.5 * (0.25 + s2 + s)
    a0 = 1.0 - a1 - a2
    return i, (a0, a1, a2)


def charge_density(p, part: np.ndarray, shape) -> np.ndarray:
    """rho(n1p, n2p, n3p) of the records part(np, ndv) (absolute positions in
    um, packed slot in the last column) with the qden weights."""
    ndim = int(p.ndim)
    n1p, n2p, n3p = shape
    rho = np.zeros(n1p * n2p * n3p, dtype=np.float64)
    if part.shape[0] == 0:
        return rho.reshape(shape, order="F")
    charge, _, wgh = unpack_slot(part[:, -1])
    w = (charge.astype(np.float32) * wgh.astype(np.float32)).astype(np.float64)
    ix, ax = _qden(p.dx_inv * (part[:, 0] - p.xmn))
    iy, ay = _qden(p.dy_inv * (part[:, 1] - p.ymn))
    if ndim == 3:
        iz, az = _qden(p.dz_inv * (part[:, 2] - p.zmn))
        zr = range(3)
    else:
        iz, az = np.ones_like(ix), (np.ones_like(w),)
        zr = range(1)
    for k1 in zr:
        kk = (iz - 1 + k1 - 1) if ndim == 3 else np.zeros_like(iz)
        for j1 in range(3):
            wy = w * ay[j1] * az[k1]
            jj = iy - 1 + j1 - 1
            for i1 in range(3):
                ii = ix - 1 + i1 - 1
                idx = ii + n1p * (jj + n2p * kk)
                rho += np.bincount(idx, weights=wy * ax[i1], minlength=rho.size)
    return rho.reshape(shape, order="F")


def step_residual(p, part0: np.ndarray, part1: np.ndarray, jc: np.ndarray, margin: int = 0):
    """Continuity residual of one step: part0 / part1 the records before /
    after it (the same particles, none removed), jc the normalised currents
    of the step (n1p, n2p, n3p, curr_ndim).  Returns (max |residual|,
    max |rho0|, max |c div J|) over the nodes at least ``margin`` nodes away
    from the array edges."""
    ndim = int(p.ndim)
    shape = jc.shape[:3]
    rho0 = charge_density(p, part0, shape)
    rho1 = charge_density(p, part1, shape)
    c = 0.5 if ndim == 2 else 1.0 / 3.0
    div = np.zeros(shape)
    for a in range(ndim):
        raw = jc[..., a] / p.djc[a]
        div += raw - np.roll(raw, 1, axis=a)
    res = (rho1 - rho0) + c * div
    if margin > 0:
        sl = tuple(slice(margin, n - margin) if (a < ndim) else slice(None) for a, n in enumerate(shape))
        res, rho0, div = res[sl], rho0[sl], div[sl]
    return float(np.abs(res).max()), float(np.abs(rho0).max()), float(np.abs(c * div).max())
