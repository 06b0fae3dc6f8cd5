"""Host-side initial laser fields (numpy), the mirror of the device's
``agpu_init_lp_fields`` / ``agpu_init_laser``, for hosts that build ``ebf``
themselves (and for the CPU runs that must start from the same pulse).

``lp_pulse(las)`` derives the arguments of the reference's
init_lp_inc0_fields from the namelist quantities, as lp_pulse
(src/IO/init_laser_field.f90:33-100) and set_initial_param
(src/start/set_init_param.f90:291-330) do for a Gaussian (g_prof) pulse:
ee0 = a0 * oml, oml = 2 pi / lam0, w0_x = tau_fwhm / sqrt(2 ln 2),
xf = focus, t0_lp = xf - xc.

``lp_fields(p, pulse)`` is init_lp_inc0_fields (src/fields/
init_grid_fields.f90:992-1386) for lp = 1: get_laser_gprof_fields_lp /
get_laser_fields_lp (487-578) in 3D and the 2D forms (406-485), each
component at its staggered position on the interior nodes, x = xmn +
(i-3) dx, xh = x + dx/2, y and z alike, in the reference's order of
operations.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import AgpuLpPulse
from .config import dims


def lp_pulse(las, g_prof: bool = True) -> AgpuLpPulse:
    a = AgpuLpPulse()
    a.om0 = 2.0 * math.pi / las.lam0
    a.ee0 = las.a0 * a.om0
    a.wx = las.tau_fwhm / math.sqrt(2. * math.log(2.)) if g_prof else \
        las.tau_fwhm / (2. * math.acos(math.sqrt(0.5 * math.sqrt(2.))) / math.pi)
    a.wy = las.w0_y
    a.xf0 = las.xf
    a.tf = las.xf - las.xc
    a.t_loc = 0.0
    a.ycent, a.zcent = las.y0, las.z0
    a.g_prof = 1 if g_prof else 0
    return a


def _fields(ndim, g_prof, par, cx, cy, cz, t1):
    """(Ex, Ey, Bx, Bz) terms of get_laser[_gprof]_fields_lp (ndim = 3) or the
    2D forms, elementwise over the coordinate arrays."""
    pi = math.acos(-1.0)
    om0, _, wx, wy, zra, eps = par
    x1 = cx
    y1 = cy / wy
    z1 = cz / wy if ndim == 3 else 0.0
    r2 = y1 * y1 + z1 * z1 if ndim == 3 else y1 * y1
    phi0 = om0 * (t1 - x1)
    if g_prof:
        phi1 = (t1 - x1) / wx
    else:
        phi1 = pi * (t1 - x1) / wx
        phi1 = np.where(np.abs(phi1) > 0.5 * pi, 0.5 * pi, phi1)
    x1 = x1 / zra
    w2 = 1. / (1. + x1 * x1)
    phx = np.arctan(x1) if ndim == 3 else 0.5 * np.arctan(x1)
    phig00 = phi0 + phx - x1 * r2 * w2
    phig10 = phig00 + phx
    tshape = np.exp(-phi1 * phi1) if g_prof else np.cos(phi1) * np.cos(phi1)
    wshape = (np.sqrt(w2) if ndim == 3 else np.sqrt(np.sqrt(w2))) * np.exp(-w2 * r2)
    ey = wshape * (tshape * np.sin(phig00))
    if g_prof and ndim == 3:
        ampl_1 = 2. * eps * tshape * w2 * np.exp(-w2 * r2)
    else:
        ampl_1 = tshape * 2. * eps * w2 * np.exp(-w2 * r2)
    ex = y1 * ampl_1 * np.cos(phig10)
    bx = z1 * ampl_1 * np.cos(phig10) if ndim == 3 else 0.0 * ex
    return ex, ey, bx


def lp_fields(p, pulse: AgpuLpPulse, ebf: np.ndarray | None = None) -> np.ndarray:
    n1p, n2p, n3p = dims(p)
    if ebf is None:
        ebf = np.zeros((n1p, n2p, n3p, p.nfield), dtype=np.float64, order="F")
    ndim = int(p.ndim)
    par = (pulse.om0, pulse.xf0 - pulse.tf, pulse.wx, pulse.wy, 0.5 * pulse.om0 * pulse.wy * pulse.wy,
           1. / (pulse.om0 * pulse.wy))
    t1 = pulse.t_loc - pulse.tf
    g = bool(pulse.g_prof)
    i = np.arange(3, p.nx + 3, dtype=np.float64)
    j = np.arange(3, p.ny + 3, dtype=np.float64)
    xx = p.xmn + p.dx * (i - 3)
    xxh = xx + 0.5 * p.dx
    yy = p.ymn + p.dy * (j - 3)
    yyh = yy + 0.5 * p.dy
    if ndim == 3:
        k = np.arange(3, p.nz + 3, dtype=np.float64)
        zz = p.zmn + p.dz * (k - 3)
        zzh = zz + 0.5 * p.dz
        sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2))

        def at(xv, yv, zv):
            X, Y, Z = np.meshgrid(xv - pulse.xf0, yv - pulse.ycent, zv - pulse.zcent, indexing="ij")
            return _fields(3, g, par, X, Y, Z, t1)

        ebf[sl + (0,)] += pulse.ee0 * at(xxh, yy, zz)[0]
        ebf[sl + (1,)] += pulse.ee0 * at(xx, yyh, zz)[1]
        ebf[sl + (3,)] += pulse.ee0 * at(xx, yyh, zzh)[2]
        ebf[sl + (5,)] += pulse.ee0 * at(xxh, yyh, zz)[1]
        # Ez(xx, yy, zzh) and By(xxh, yy, zzh) are zero for this polarisation
    else:
        sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(0, 1))

        def at(xv, yv):
            X, Y = np.meshgrid(xv - pulse.xf0, yv - pulse.ycent, indexing="ij")
            return tuple(f[..., None] for f in _fields(2, g, par, X, Y, 0.0, t1))

        ebf[sl + (0,)] += pulse.ee0 * at(xxh, yy)[0]
        ebf[sl + (1,)] += pulse.ee0 * at(xx, yyh)[1]
        ebf[sl + (2,)] += pulse.ee0 * at(xxh, yyh)[1]
    return ebf


def laser_fields(p, las) -> np.ndarray:
    """ebf with the Gaussian pulse of ``las`` (an AgpuLaser), as agpu_init_laser
    sets it on the device."""
    return lp_fields(p, lp_pulse(las, True))
