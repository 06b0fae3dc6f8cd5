"""A known answer for the oracle's field solver: the numerical dispersion of
the leapfrog Yee scheme (advance_lpf_fields with rote / rotb,
src/dynamics/curr_and_fields_util.f90:176-260, src/fields/grid_fields.f90:
1405-1552) with the x difference of se_coeff (src/fields/
grid_field_param.f90:54-97).

A plane-wave mode exp(i (k.x - w t)) of that scheme obeys

    sin(w dt / 2)^2 / dt^2 = Kx^2 + Ky^2 (+ Kz^2),
    Kx = (c1 sin(kx dx / 2) + c2 sin(3 kx dx / 2)) / dx,
    Ky = sin(ky dy / 2) / dy,  Kz = sin(kz dz / 2) / dz,

with (c1, c2) = se_coeff: (1, 0) for der_ord 2.  A vacuum pulse's energy
centroid moves at the group velocity dw/dkx averaged over its energy
spectrum.  The test launches a Gaussian pulse (carrier 0.8 um on a grid of
10 cells per um, where the second-order scheme is 3-4 % slower than c) and
checks the centroid's speed after a few hundred steps against that
prediction, computed from the initial field's discrete spectrum, to 1 % of
the predicted slowdown; the third-order x difference cuts the slowdown
several fold, as its coefficients are meant to."""
import math

import numpy as np
import pytest

from aladyn_b200.config import Grid, dims, make_params
from oracle.oracle import Oracle

LAM = 0.8


def _pulse(p, xc, length, w0):
    """Ey(i, j+1/2, k) and Bz(i+1/2, j+1/2, k) = Ey of a forward pulse."""
    n1p, n2p, n3p = dims(p)
    nf = p.nfield
    ebf = np.zeros((n1p, n2p, n3p, nf), order="F")
    x = p.xmn + (np.arange(1, n1p + 1) - 3) * p.dx
    yh = p.ymn + (np.arange(1, n2p + 1) - 3 + 0.5) * p.dy
    z = p.zmn + (np.arange(1, n3p + 1) - 3) * p.dz if p.ndim == 3 else np.zeros(1)
    kl = 2 * math.pi / LAM

    def ey(xv):
        X, Y, Z = np.meshgrid(xv, yh, z, indexing="ij")
        return np.exp(-((X - xc) / length) ** 2 - (Y ** 2 + Z ** 2) / w0 ** 2) * np.cos(kl * (X - xc))

    ebf[..., 1] = ey(x)
    ebf[..., nf - 1] = ey(x + 0.5 * p.dx)
    inner = np.zeros((n1p, n2p, n3p), dtype=bool)
    inner[2:p.nx + 2, 2:p.ny + 2, _ks(p)] = True
    for c in range(nf):
        ebf[..., c] = np.where(inner, ebf[..., c], 0.0)
    return ebf, x


def _ks(p):
    return slice(2, p.nz + 2) if p.ndim == 3 else slice(0, 1)


def _centroid(p, f, x):
    ks, nf = _ks(p), p.nfield
    xi = x[2:p.nx + 2]
    we = (f[2:p.nx + 2, 2:p.ny + 2, ks, 1] ** 2).sum(axis=(1, 2))
    wb = (f[2:p.nx + 2, 2:p.ny + 2, ks, nf - 1] ** 2).sum(axis=(1, 2))
    return ((xi * we).sum() + ((xi + 0.5 * p.dx) * wb).sum()) / (we.sum() + wb.sum())


def _predicted(p, ey0):
    """Group velocity dw/dkx averaged over |FFT(Ey)|^2."""
    spec = np.abs(np.fft.fftn(ey0)) ** 2
    ax = [np.abs(2 * math.pi * np.fft.fftfreq(n, d)) for n, d in zip(ey0.shape, (p.dx, p.dy, p.dz))]
    kx, ky, kz = np.meshgrid(*ax, indexing="ij")
    c1, c2 = p.se_coeff[0], p.se_coeff[1]

    def omega(k):
        kx2 = ((c1 * np.sin(k * p.dx / 2) + c2 * np.sin(3 * k * p.dx / 2)) / p.dx) ** 2
        ky2 = (np.sin(ky * p.dy / 2) / p.dy) ** 2
        kz2 = (np.sin(kz * p.dz / 2) / p.dz) ** 2 if p.ndim == 3 else 0.0
        return 2 / p.dt * np.arcsin(p.dt * np.sqrt(kx2 + ky2 + kz2))

    h = 1e-5
    vg = (omega(kx + h) - omega(kx - h)) / (2 * h)
    return float((spec * vg).sum() / spec.sum())


def _measure(ndim, der_ord, nx, ntr, steps, length, w0, w_sh=0, shifts=None):
    g = Grid(ndim, nx, ntr, ntr, k0=10.0, yx_rat=4.0, zx_rat=4.0, cfl=0.8)
    p = make_params(g, w_sh=w_sh, capacity=(16, 0, 0, 0), der_ord=der_ord)
    ebf, x = _pulse(p, p.xmn + 0.25 * nx * p.dx, length, w0)
    o = Oracle(p)
    o.set_fields(ebf)
    c0 = _centroid(p, o.get_fields(), x)
    t = 0.0
    for it in range(steps):
        rc, out = o.lp_run(t, it)
        assert rc == 0
        if shifts is not None:
            shifts.append(out.nshx)
        t += p.dt
    # lab-frame positions: the window's origin moved by the shifts
    lab = x + (o.xmn() - p.xmn)
    v = (_centroid(p, o.get_fields(), lab) - c0) / (steps * p.dt)
    return v, _predicted(p, ebf[2:nx + 2, 2:ntr + 2, _ks(p), 1])


CASES = {2: dict(nx=640, ntr=64, steps=400, length=4.0, w0=6.0),
         3: dict(nx=320, ntr=48, steps=200, length=3.0, w0=4.0)}


@pytest.mark.parametrize("ndim", [2, 3])
def test_pulse_moves_at_the_schemes_group_velocity(ndim):
    slow = {}
    for der_ord in (2, 3):
        v, vp = _measure(ndim, der_ord, **CASES[ndim])
        print(f"{ndim}D der_ord {der_ord}: measured {v:.7f} predicted {vp:.7f}")
        assert abs(v - vp) <= 0.01 * (1.0 - vp), (der_ord, v, vp)
        slow[der_ord] = 1.0 - vp
    assert slow[2] > 0.03
    assert slow[3] < slow[2] / 5


def test_group_velocity_in_the_moving_window():
    """The same 2D pulse inside the moving window (w_sh 10, w_speed 1):
    every shift moves the fields by whole cells and the origin with them,
    so the lab-frame centroid still moves at the group velocity, and the
    window has advanced by the rounded lapse nint(dx_inv * w_speed * dt *
    w_sh * shifts) cells (lp_window_xshift, src/dynamics/window.f90:
    276-347), while the pulse (slower than c) slid back in the window."""
    shifts = []
    v, vp = _measure(2, 2, **CASES[2], w_sh=10, shifts=shifts)
    # a shift at every iteration 10, 20, ... 390 of the 400
    nsh = [n for n in shifts if n > 0]
    assert [i for i, n in enumerate(shifts) if n > 0] == list(range(10, 400, 10))
    g = Grid(2, 640, 64, 64, k0=10.0, yx_rat=4.0, zx_rat=4.0, cfl=0.8)
    p = make_params(g, w_sh=10, capacity=(16, 0, 0, 0))
    assert sum(nsh) == round(p.dx_inv * p.dt * 10 * len(nsh))
    assert abs(v - vp) <= 0.01 * (1.0 - vp), (v, vp)


@pytest.mark.parametrize("ndim", [2, 3])
def test_open_boundary_absorbs_the_outgoing_pulse(ndim):
    """The open x boundary (the Mur-type ef_bds / bf_bds faces, src/fields/
    grid_fields.f90:1069-1354) lets a pulse leave: once the pulse has run
    out through the right face, under 0.5 % of its field energy is left in
    the box (measured 0.05 % in 2D, 0.14 % in 3D; a reflecting face would
    keep all of it)."""
    nx, ntr = (400, 64) if ndim == 2 else (200, 40)
    g = Grid(ndim, nx, ntr, ntr, k0=10.0, yx_rat=4.0, zx_rat=4.0, cfl=0.8)
    p = make_params(g, w_sh=0, capacity=(16, 0, 0, 0))
    lx = nx * p.dx
    ebf, _ = _pulse(p, p.xmn + 0.6 * lx, 0.12 * lx, 0.25 * ntr * p.dy)
    o = Oracle(p)
    o.set_fields(ebf)
    ks = _ks(p)

    def energy(f):
        return float((f[2:nx + 2, 2:ntr + 2, ks, :] ** 2).sum())

    e0 = energy(o.get_fields())
    t = 0.0
    for it in range(int(0.75 * lx / p.dt)):
        rc, _ = o.lp_run(t, it)
        assert rc == 0
        t += p.dt
    assert energy(o.get_fields()) < 5e-3 * e0
