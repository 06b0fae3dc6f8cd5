"""Derived simulation parameters, as ALaDyn's start-up computes them.

``make_params`` restates the subset of ``set_initial_param``
(src/start/set_init_param.f90:25-414), ``set_grid`` (src/grid/
set_grid_param.f90:52-226), ``set_fyzxgrid`` / ``set_loc_grid_param``
(set_grid_param.f90:473-662, 811-829) and ``set_field_param``
(src/fields/grid_field_param.f90:36-99) that the PIC step reads, for one
domain (one GPU), a uniform grid and open boundaries.  Python floats are
IEEE doubles, and each expression keeps the Fortran evaluation order so the
values are bit-identical to what the reference computes with
-fdefault-real-8.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

from .abi import AGPU_FP32_SPLIT, AGPU_FP64, AgpuLaser, AgpuParams, AgpuPlasma

PI = 3.141592653589793          # src/work/phys_param.f90:27
RC0 = 2.81794033                # phys_param.f90:49
REFERENCE_DENSITY = 1.e6        # phys_param.f90:57
PROTON_MASS_NORM = 1836.1527706  # phys_param.f90:37


@dataclass
class Grid:
    ndim: int
    nx: int
    ny: int
    nz: int
    k0: float          # grid points per micron along x (dx = 1/k0)
    yx_rat: float
    zx_rat: float
    cfl: float


def nint(x: float) -> int:
    """Fortran NINT: round half away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def ompe_value() -> float:
    """ompe = 4 pi rc0 (reference_density 1e-6) 1e-3 (set_init_param.f90:254-255)."""
    ompe = 4. * PI * RC0 * (REFERENCE_DENSITY * 1.e-6)
    return 1.e-03 * ompe


def make_params(grid: Grid, *, precision: int = AGPU_FP64, nsp: int = 1, nsp_run: int = 1,
                w_sh: int = 10, w_speed: float = 1.0, wi_time: float = 0.0,
                wf_time: float = 1.0e9, capacity=(0, 0, 0, 0), der_ord: int = 2,
                mass_number=(1.0, 1.0, 1.0), ionz_lev: int = 0, n_mol_atoms=(1, 1, 1, 1),
                seed: int = 12345, shape: int = 0, iform: int = 0) -> AgpuParams:
    p = AgpuParams()
    ndim = grid.ndim
    p.ndim = ndim
    p.nx, p.ny = grid.nx, grid.ny
    p.nz = grid.nz if ndim == 3 else 1
    p.nfield = 6 if ndim == 3 else 3
    p.curr_ndim = 3 if ndim == 3 else 2
    p.ibx = p.iby = p.ibz = 0
    p.iform = iform  # 0, 1: charge-conserving Esirkepov deposit; 2: ncdef (FP64 form)
    p.precision = precision
    p.nsp = nsp
    p.nsp_run = nsp_run
    p.w_sh = w_sh
    p.ionz_lev = ionz_lev
    p.shape = shape  # 0: the reference's quadratic/linear shapes, 1: cubic extension
    for i in range(4):
        p.n_mol_atoms[i] = n_mol_atoms[i]
    # set_grid (set_grid_param.f90:52-226), uniform axes
    dx = 1. / grid.k0
    dx_inv = 1.0 / dx
    dy = grid.yx_rat * dx
    dy_inv = 1. / dy
    dz, dz_inv = 1., 1.
    if ndim == 3:
        dz = grid.zx_rat * dx
        dz_inv = 1. / dz
    p.dx, p.dy, p.dz = dx, dy, dz
    p.dx_inv, p.dy_inv, p.dz_inv = dx_inv, dy_inv, dz_inv
    # dt (set_init_param.f90:79-89)
    if ndim == 2:
        p.dt = grid.cfl / math.sqrt(dx_inv * dx_inv + dy_inv * dy_inv)
    else:
        p.dt = grid.cfl / math.sqrt(dx_inv * dx_inv + dy_inv * dy_inv + dz_inv * dz_inv)
    # x(i) = dx*(i-1), y(i) = dy*(i-1-ny/2), z(i) = dz*(i-1-nz/2)
    def xg(i): return dx * float(i - 1)
    def yg(i): return dy * float(i - 1 - grid.ny // 2)
    def zg(i): return dz * float(i - 1 - grid.nz // 2)
    p.xmn, p.gxmin, p.gxmax = xg(1), xg(1), xg(grid.nx + 1)
    p.xmax = xg(grid.nx)
    p.ymn, p.gymin, p.gymax = yg(1), yg(1), yg(grid.ny + 1)
    if ndim == 3:
        p.zmn, p.gzmin, p.gzmax = zg(1), zg(1), zg(grid.nz + 1)
    else:
        p.zmn, p.gzmin, p.gzmax = 0.0, 0.0, 0.0
    # set_field_param (grid_field_param.f90:36-99)
    if der_ord == 2:
        p.se_coeff[0], p.se_coeff[1] = 1., 0.
    elif der_ord == 3:
        nu = grid.cfl * grid.yx_rat / math.sqrt(grid.yx_rat * grid.yx_rat + float(ndim) - 1.)
        c1 = 1. + 0.125 * (1. - nu * nu)
        p.se_coeff[0], p.se_coeff[1] = c1, (1. - c1) / 3.
    else:
        raise ValueError("der_ord must be 2 or 3")
    # djc (set_init_param.f90:92-103)
    if ndim == 2:
        p.djc[0], p.djc[1], p.djc[2] = 0.5 * dx, 0.5 * dy, 0.0
    else:
        p.djc[0], p.djc[1], p.djc[2] = dx / 3., dy / 3., dz / 3.
    p.ompe = ompe_value()
    # lorentz_fact = 1/mass (set_init_param.f90:196-206)
    masses = [1.0] + [m * PROTON_MASS_NORM for m in mass_number]
    for i in range(4):
        p.lorentz_fact[i] = 1. / masses[i]
    p.w_speed, p.wi_time, p.wf_time = w_speed, wi_time, wf_time
    p.seed = seed
    for i in range(4):
        p.capacity[i] = int(capacity[i])
    return p


class StretchedGrid:
    """The stretched transverse axes of set_grid (src/grid/set_grid_param.f90:
    52-226) with str_flag 1 or 2 (set_init_param.f90:54-69): ny_stretch =
    nint(ny/6) (1) or nint(ny/4) (2) cells at each end of y (and z in 3D,
    nz_stretch = ny_stretch) follow y = s + L tan(xi) on a uniform xi grid of
    step dxi = 0.4 pi / ny_stretch, L = dy / dxi.  Holds the node
    coordinates y, yh (0 .. n+1), the metric factors d1 = cos^2(xi) and d1h
    (the reference's dy1, dy1h, loc_yg(:, 3:4)) and the agpu_stretch struct
    for the library and the oracle."""

    def __init__(self, p: "AgpuParams", str_flag: int = 1):
        import numpy as np

        from .abi import AgpuStretch
        if p.ndim < 2 or str_flag not in (1, 2):
            raise ValueError("stretched grids need ndim >= 2 and str_flag 1 or 2")
        size = float(np.float32(1.0) / np.float32(6.0))  # size_of_stretch_along_y = 1./6. (default real)
        f = float(p.ny) * size if str_flag == 1 else float(p.ny) * 1.5 * size
        self.n_stretch = int(math.floor(f + 0.5))  # nint
        # aph = acos(-1.0)*0.4 in default real
        self.aph = float(np.float32(np.arccos(np.float32(-1.0))) * np.float32(0.4))
        self.st = AgpuStretch()
        self.st.on = 1
        self.y = self._axis(p.ny, p.dy, p.dy_inv, self.st.y)
        if p.ndim == 3:
            self.z = self._axis(p.nz, p.dz, p.dz_inv, self.st.z)
        # loc_ygrid / loc_zgrid bounds: gmin = y(1), gmax = y(n+1)
        p.ymn = p.gymin = self.y["y"][1]
        p.gymax = self.y["y"][p.ny + 1]
        if p.ndim == 3:
            p.zmn = p.gzmin = self.z["y"][1]
            p.gzmax = self.z["y"][p.nz + 1]
        self.struct = self.st

    def _axis(self, n, d, d_inv, ax):
        import numpy as np
        ys = self.n_stretch
        y = [d * float(i - 1 - n // 2) for i in range(n + 2)]
        yh = [v + 0.5 * d for v in y]
        d1 = [1.0] * (n + 2)
        d1h = [1.0] * (n + 2)
        ns1 = n + 1 - ys
        dli = self.aph / float(ys)
        dli_inv = 1. / dli
        l_s = d * dli_inv
        ratio = dli * d_inv
        smin, smax = y[ys + 1], y[ns1]
        for i in range(0, ys + 1):
            yy = dli * float(i - 1 - ys)
            yyh = yy + 0.5 * dli
            y[i] = smin + l_s * math.tan(yy)
            yh[i] = smin + l_s * math.tan(yyh)
            d1h[i] = math.cos(yyh) * math.cos(yyh)
            d1[i] = math.cos(yy) * math.cos(yy)
        for i in range(ns1, n + 2):
            yy = dli * float(i - ns1)
            yyh = yy + dli * 0.5
            y[i] = smax + l_s * math.tan(yy)
            yh[i] = smax + l_s * math.tan(yyh)
            d1h[i] = math.cos(yyh) * math.cos(yyh)
            d1[i] = math.cos(yy) * math.cos(yy)
        out = {"y": np.array(y), "yh": np.array(yh), "d1": np.ascontiguousarray(d1, dtype=np.float64),
               "d1h": np.ascontiguousarray(d1h, dtype=np.float64), "smin": smin, "smax": smax, "l_s": l_s,
               "dli": dli}
        # map2dy_part_sind's parameters (stretched_grid.f90:80-88)
        ax.cnst = 1.0 * n * d / 2
        ax.smin, ax.smax = smin, smax
        ax.xs = ys * d
        ax.dl_inv = d_inv
        ax.dli_inv = dli_inv
        ax.ratio = ratio
        ax.nl_stretch = float(ys)
        ax.init_cell = 0.0
        ax.n = n
        ax.d1 = out["d1"].ctypes.data_as(C.POINTER(C.c_double))
        ax.d1h = out["d1h"].ctypes.data_as(C.POINTER(C.c_double))
        return out

    def map(self, axis: str, v: float) -> float:
        """The particle map of the axis (the library's str_map), in Python."""
        a = self.st.y if axis == "y" else self.st.z
        def inv(yp):
            return a.dli_inv * math.atan(a.ratio * (yp + a.cnst - a.xs)) + a.nl_stretch
        if v <= a.smin:
            return inv(v) - a.init_cell
        if v >= a.smax:
            return (a.n - inv(2 * 0.0 - v)) - a.init_cell
        return (v + a.cnst) * a.dl_inv - a.init_cell


def env_params(grid: Grid, lam0: float, der_ord: int = 2):
    """The envelope solver's constants: oml = 2 pi / lam0 and, for der_ord 3,
    opt_der1 = (4 - nu^2)/3 and hord_der2 = -(1 - nu^2)/12 with the
    multi-D optimised nu of set_field_param (grid_field_param.f90:36-72)."""
    from .abi import AgpuEnvParams
    e = AgpuEnvParams()
    e.om0 = 2.0 * PI / lam0
    e.der_ord = der_ord
    e.opt_der1, e.hord_der2 = 1.0, 0.0
    if der_ord == 3:
        nu = grid.cfl
        if grid.ndim > 1:
            nu = grid.cfl * grid.yx_rat / math.sqrt(grid.yx_rat * grid.yx_rat + float(grid.ndim) - 1.)
        e.hord_der2 = -(1. - nu * nu) / 12.
        e.opt_der1 = (4. - nu * nu) / 3.
    elif der_ord != 2:
        raise ValueError("der_ord must be 2 or 3")
    return e


def n_over_nc_to_n0(n_over_nc: float, lam0: float) -> float:
    """n0_ref (1e18 cm^-3) giving electron density n/nc (set_init_param.f90:272-279)."""
    ncrit = PI / (RC0 * lam0 * lam0)
    return n_over_nc * ncrit / 1.e-03


def plasma(ic: int, npx: int, npy: int, npz: int, charge: int, wgh: float, x_start: float,
           x_end: float, y_min: float, y_max: float, z_min: float = 0.0, z_max: float = 0.0,
           jitter: float = 0.5, seed: int = 2024, part_ind: int = 0) -> AgpuPlasma:
    s = AgpuPlasma()
    s.ic, s.npx, s.npy, s.npz = ic, npx, npy, npz
    s.charge, s.part_ind, s.wgh = charge, part_ind, wgh
    s.x_start, s.x_end = x_start, x_end
    s.y_min, s.y_max, s.z_min, s.z_max = y_min, y_max, z_min, z_max
    s.jitter = jitter
    s.seed = seed
    return s


def laser(a0: float, lam0: float, w0_y: float, tau_fwhm: float, xc: float, xf: float,
          y0: float = 0.0, z0: float = 0.0) -> AgpuLaser:
    l = AgpuLaser()
    l.a0, l.lam0, l.w0_y, l.tau_fwhm, l.xc, l.xf, l.y0, l.z0 = a0, lam0, w0_y, tau_fwhm, xc, xf, y0, z0
    return l


def dims(p: AgpuParams):
    """(n1p, n2p, n3p): allocated field extents (array_alloc.f90:63-71)."""
    return p.nx + 5, p.ny + 5, (p.nz + 5 if p.ndim == 3 else 1)


def ndv(p: AgpuParams) -> int:
    return 7 if p.ndim == 3 else 5


__all__ = ["Grid", "make_params", "plasma", "laser", "dims", "ndv", "nint", "ompe_value", "env_params",
           "n_over_nc_to_n0", "AGPU_FP64", "AGPU_FP32_SPLIT"]
