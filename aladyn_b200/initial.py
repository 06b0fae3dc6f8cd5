"""Host-side initial laser fields (numpy), the mirror of the device
``agpu_init_laser`` kernel, for hosts that build ``ebf`` themselves.

Linearly polarised (y) paraxial Gaussian pulse moving along +x: Ey on
(i, j+1/2, k), Bz = Ey(x + dx/2) on (i+1/2, j+1/2, k), both at t = 0, with the
longitudinal envelope exp(-((x-xc)/w0_x)^2), w0_x = tau_fwhm/sqrt(2 ln 2), as
the reference's Gaussian (g_prof) pulse (src/start/set_init_param.f90:318-330).
"""
from __future__ import annotations

import math

import numpy as np

from .config import dims


def laser_fields(p, las) -> np.ndarray:
    n1p, n2p, n3p = dims(p)
    ebf = np.zeros((n1p, n2p, n3p, p.nfield), dtype=np.float64, order="F")
    k0 = 2.0 * math.pi / las.lam0
    amp = las.a0 * k0
    w0 = las.w0_y
    zr = math.pi * w0 * w0 / las.lam0
    w0x = las.tau_fwhm / math.sqrt(2.0 * math.log(2.0))
    ii = np.arange(3, p.nx + 3)
    jj = np.arange(3, p.ny + 3)
    kk = np.arange(3, p.nz + 3) if p.ndim == 3 else np.array([3])
    x = p.xmn + (ii - 3) * p.dx
    y = p.ymn + (jj - 3 + 0.5) * p.dy
    z = p.zmn + (kk - 3) * p.dz if p.ndim == 3 else np.zeros(1)

    def ey(xv):
        X, Y, Z = np.meshgrid(xv, y, z, indexing="ij")
        xi = X - las.xf
        wr = w0 * np.sqrt(1.0 + (xi / zr) ** 2)
        r2 = (Y - las.y0) ** 2 + ((Z - las.z0) ** 2 if p.ndim == 3 else 0.0)
        rinv = xi / (xi * xi + zr * zr)
        gouy = np.arctan(xi / zr)
        a = (w0 / wr) if p.ndim == 3 else np.sqrt(w0 / wr)
        ph = k0 * (X - las.xc) + 0.5 * k0 * r2 * rinv - (gouy if p.ndim == 3 else 0.5 * gouy)
        ex = (X - las.xc) / w0x
        return amp * a * np.exp(-r2 / (wr * wr)) * np.exp(-ex * ex) * np.cos(ph)

    sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2) if p.ndim == 3 else slice(0, 1))
    ebf[sl + (1,)] = ey(x)
    ebf[sl + (p.nfield - 1,)] = ey(x + 0.5 * p.dx)
    return ebf
