"""Shared small LWFA cases for the tests: parameters, a laser pulse on the
staggered grid (numpy, fed identically to the oracle and the device) and the
lattice plasma source."""
from __future__ import annotations

import math

import numpy as np

from aladyn_b200.config import Grid, dims, laser, make_params, plasma
from aladyn_b200.abi import AGPU_FP64

LAM0 = 0.8


def grid_small(ndim, nx=64, ny=32, nz=16):
    if ndim == 2:
        return Grid(2, nx, ny, 1, k0=25.0, yx_rat=4.0, zx_rat=1.0, cfl=0.8)
    return Grid(3, nx, ny, nz, k0=25.0, yx_rat=5.0, zx_rat=5.0, cfl=0.8)


def laser_fields(p, a0=2.0, w0=None, tau=None, xc=None, xf=None, dtype=np.float64):
    """Ey on (i, j+1/2, k) and Bz on (i+1/2, j+1/2, k) of a linearly
    polarised Gaussian pulse (paraxial, envelope exp(-((x-xc)/w0x)^2)) plus a
    small static Ex/Ez/Bx/By pattern so every component is exercised."""
    n1p, n2p, n3p = dims(p)
    nf = p.nfield
    ebf = np.zeros((n1p, n2p, n3p, nf), dtype=dtype, order="F")
    Lx = p.nx * p.dx
    w0 = w0 if w0 is not None else 0.25 * p.ny * p.dy
    tau = tau if tau is not None else 0.3 * Lx
    xc = xc if xc is not None else 0.55 * Lx
    xf = xf if xf is not None else xc
    k0 = 2 * math.pi / LAM0
    amp = a0 * k0
    w0x = tau / math.sqrt(2 * math.log(2))
    i = np.arange(1, n1p + 1)
    j = np.arange(1, n2p + 1)
    k = np.arange(1, n3p + 1)
    x = p.xmn + (i - 3) * p.dx
    yh = p.ymn + (j - 3 + 0.5) * p.dy
    y = p.ymn + (j - 3) * p.dy
    z = (p.zmn + (k - 3) * p.dz) if p.ndim == 3 else np.zeros(1)
    zh = (p.zmn + (k - 3 + 0.5) * p.dz) if p.ndim == 3 else np.zeros(1)

    def ey(xv, yv, zv):
        X, Y, Z = np.meshgrid(xv, yv, zv, indexing="ij")
        r2 = Y ** 2 + (Z ** 2 if p.ndim == 3 else 0.0)
        env = np.exp(-((X - xc) / w0x) ** 2) * np.exp(-r2 / w0 ** 2)
        return amp * env * np.cos(k0 * (X - xc))

    ebf[..., 1] = ey(x, yh, z)                      # Ey(i, j+1/2, k)
    ebf[..., nf - 1] = ey(x + 0.5 * p.dx, yh, z)    # Bz(i+1/2, j+1/2, k)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    ebf[..., 0] = 0.05 * amp * np.sin(2 * math.pi * X / Lx) * np.cos(Y / (p.ny * p.dy))
    if nf == 6:
        ebf[..., 2] = 0.03 * amp * np.cos(2 * math.pi * X / Lx) * np.sin(2 * Z / (p.nz * p.dz) + 0.3)
        ebf[..., 3] = 0.02 * amp * np.sin(2 * math.pi * X / Lx + 0.7)
        ebf[..., 4] = 0.02 * amp * np.cos(2 * math.pi * X / Lx + 0.1) * np.cos(Y / (p.ny * p.dy))
    # zero the frame outside the interior, as the reference's loaders leave it
    mask = np.zeros_like(ebf[..., 0], dtype=bool)
    mask[2:p.nx + 2, 2:p.ny + 2, (2 if p.ndim == 3 else 0):(p.nz + 2 if p.ndim == 3 else 1)] = True
    for c in range(nf):
        ebf[..., c] = np.where(mask, ebf[..., c], 0.0)
    return ebf


def plasma_source(p, ic=0, npx=2, npy=2, npz=2, x_start_frac=0.25, jitter=0.6, seed=777,
                  charge=-1, wgh=None, n_over_n0=17.42):
    ppc = npx * npy * (npz if p.ndim == 3 else 1)
    w = wgh if wgh is not None else n_over_n0 / ppc
    return plasma(ic, npx, npy, npz if p.ndim == 3 else 1, charge, w,
                  x_start=p.gxmin + x_start_frac * p.nx * p.dx, x_end=1.0e6,
                  y_min=p.gymin + 2 * p.dy, y_max=p.gymax - 2 * p.dy,
                  z_min=(p.gzmin + 2 * p.dz) if p.ndim == 3 else 0.0,
                  z_max=(p.gzmax - 2 * p.dz) if p.ndim == 3 else 0.0,
                  jitter=jitter, seed=seed)


def small_case(ndim, precision=AGPU_FP64, nx=64, ny=32, nz=16, cap=200_000, w_sh=10, nsp=1,
               ionz_lev=0, n_mol_atoms=(1, 1, 1, 1), seed=12345, iform=0):
    g = grid_small(ndim, nx, ny, nz)
    p = make_params(g, precision=precision, nsp=nsp, nsp_run=1, w_sh=w_sh,
                    capacity=(cap, cap if nsp > 1 else 0, cap if nsp > 2 else 0, 0),
                    ionz_lev=ionz_lev, n_mol_atoms=n_mol_atoms, seed=seed,
                    mass_number=(14.0, 1.0, 1.0), iform=iform)
    return p


def sort_records(a: np.ndarray) -> np.ndarray:
    """Order-independent view of a particle set (lexicographic by all columns)."""
    if a.shape[0] == 0:
        return a
    idx = np.lexsort(a.T[::-1])
    return a[idx]


# ---- PWFA bunch (the 512x256x256 PWFA set-up on small grids) ----------------
def grid_pwfa(ndim, nx=48, ny=32, nz=32):
    """dx = 0.2 um, dy = dz = 0.5 um as the 512x256x256 PWFA case."""
    if ndim == 2:
        return Grid(2, nx, ny, 1, k0=5.0, yx_rat=2.5, zx_rat=1.0, cfl=0.8)
    return Grid(3, nx, ny, nz, k0=5.0, yx_rat=2.5, zx_rat=2.5, cfl=0.8)


def pwfa_bunch(p, nb=20000, sxb=2.0, syb=1.5, gam=1957.0, seed=77):
    """A 200 pC bunch centred in the box (gam 1957, 1% spread, 1 um emittance)."""
    from aladyn_b200.beam import Bunch
    return Bunch(nb_tot=nb, charge_pc=200.0, sxb=sxb, syb=syb, gam=gam, epsy=1.0, epsz=1.0, dg=1.0,
                 xc=p.xmn + 0.5 * p.nx * p.dx, yc=0.0, zc=0.0, seed=seed)


def sine_mode(p, n1p, n2p, n3p, a, b, c):
    """rho with a pure DST-I mode (a, b, c) (0-based) on the interior."""
    n1, n2, n3 = p.nx, p.ny, (p.nz if p.ndim == 3 else 1)
    sx = np.sin(np.pi * np.arange(1, n1 + 1) * (a + 1) / (n1 + 1))
    sy = np.sin(np.pi * np.arange(1, n2 + 1) * (b + 1) / (n2 + 1))
    sz = np.sin(np.pi * np.arange(1, n3 + 1) * (c + 1) / (n3 + 1)) if p.ndim == 3 else np.ones(1)
    rho = np.zeros((n1p, n2p, n3p), order="F")
    k0 = 2 if p.ndim == 3 else 0
    rho[2:2 + n1, 2:2 + n2, k0:k0 + n3] = sx[:, None, None] * sy[None, :, None] * sz[None, None, :]
    return rho


def sine_mode_potential(p, rho, a, b, c, gam2):
    """The reference solver's answer for a pure mode: omp0 rho / k^2 with
    k_i = 2 sin(d_i ak_i / 2)/d_i, ak = pi i / l_box, and the x round-trip
    factor (n1+1)/(n1+2) of its forward scale 1/(2(n1+2)) (3D only)."""
    def sk(d, l, i):
        return 2. * math.sin(0.5 * d * (math.acos(-1.0) / l * i)) / d
    lx, ly, lz = p.xmax - p.xmn, p.gymax - p.gymin, p.gzmax - p.gzmin
    if p.ndim == 3:
        ak2 = sk(p.dz, lz, c + 1) ** 2 + sk(p.dy, ly, b + 1) ** 2 + sk(p.dx, lx, a + 1) ** 2 / gam2
        return rho * (p.ompe / ak2) * (p.nx + 1) / (p.nx + 2)
    return rho * (p.ompe / sk(p.dy, ly, b + 1) ** 2)


def inside_box(p, rec):
    """The records mpi_beam_distribute keeps: gxmin < x <= gxmax, y and z alike."""
    m = (rec[:, 0] > p.gxmin) & (rec[:, 0] <= p.gxmax) & (rec[:, 1] > p.gymin) & (rec[:, 1] <= p.gymax)
    if p.ndim == 3:
        m &= (rec[:, 2] > p.gzmin) & (rec[:, 2] <= p.gzmax)
    return rec[m]
