"""The laser set-up restated from the reference (init_lp_inc0_fields with
get_laser_gprof_fields_lp / get_laser_fields_lp and their 2D forms,
src/fields/init_grid_fields.f90:406-578, 992-1386): the oracle's C
restatement and the host numpy one (aladyn_b200.initial, which feeds the
CPU runs) agree to round-off on every component, Gaussian and cos^2
profiles, 2D and 3D; the longitudinal Ex and Bx terms are present; the
peak of Ey at the focus is the amplitude ee0 = a0 * 2 pi / lam0."""
import math

import numpy as np
import pytest

from aladyn_b200.config import laser
from aladyn_b200.initial import lp_fields, lp_pulse
from oracle.oracle import Oracle
from tests.helpers import LAM0, small_case


def _pulse(p, g_prof, a0=2.0):
    lx = p.nx * p.dx
    las = laser(a0, LAM0, 0.3 * p.ny * p.dy, 4 * LAM0, xc=0.5 * lx, xf=0.55 * lx, y0=0.1, z0=-0.2)
    return lp_pulse(las, g_prof)


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("g_prof", [True, False])
def test_oracle_and_host_laser_agree(ndim, g_prof):
    p = small_case(ndim, nx=96, ny=48, nz=32, cap=16)
    a = _pulse(p, g_prof)
    o = Oracle(p)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    o.init_lp_fields(a)
    fo = o.get_fields()
    fh = lp_fields(p, a)
    scale = np.abs(fo).max()
    assert scale > 0
    assert np.abs(fo - fh).max() <= 1e-13 * scale
    ex, ey, bz = fo[..., 0], fo[..., 1], fo[..., p.nfield - 1]
    assert np.abs(ex).max() > 1e-3 * np.abs(ey).max()  # the longitudinal term
    if ndim == 3:
        assert np.abs(fo[..., 3]).max() > 1e-3 * np.abs(ey).max()  # Bx
        assert np.abs(fo[..., 2]).max() == 0.0 and np.abs(fo[..., 4]).max() == 0.0
    assert np.abs(bz).max() > 0.5 * np.abs(ey).max()
    # nothing outside the interior nodes
    inner = np.zeros(fo.shape[:3], dtype=bool)
    inner[2:p.nx + 2, 2:p.ny + 2, (2 if ndim == 3 else 0):(p.nz + 2 if ndim == 3 else 1)] = True
    assert np.abs(fo[~inner]).max() == 0.0


def test_peak_amplitude_at_focus():
    """A pulse centred on its focus (tf = 0): |Ey| peaks at ee0 on axis."""
    p = small_case(3, nx=160, ny=32, nz=32, cap=16)
    lx = p.nx * p.dx
    las = laser(1.5, LAM0, 2.0, 6 * LAM0, xc=0.5 * lx, xf=0.5 * lx)
    a = lp_pulse(las, True)
    f = lp_fields(p, a)
    ee0 = 1.5 * 2 * math.pi / LAM0
    assert 0.97 * ee0 <= np.abs(f[..., 1]).max() <= ee0


def _div_e(f, p):
    """Discrete div E at the nodes (i, j, k) from the staggered components."""
    d = (f[1:-1, 1:-1, :, 0] - f[:-2, 1:-1, :, 0]) / p.dx + (f[1:-1, 1:-1, :, 1] - f[1:-1, :-2, :, 1]) / p.dy
    if p.ndim == 3:
        d = d[:, :, 1:-1] + (f[1:-1, 1:-1, 1:-1, 2] - f[1:-1, 1:-1, :-2, 2]) / p.dz
    return d[3:-3, 3:-3, 3:-3] if p.ndim == 3 else d[3:-3, 3:-3]


def _div_b(f, p):
    """Discrete div B at the cell centres (i+1/2, j+1/2, k+1/2)."""
    d = ((f[2:, 1:-1, 1:-1, 3] - f[1:-1, 1:-1, 1:-1, 3]) / p.dx
         + (f[1:-1, 2:, 1:-1, 4] - f[1:-1, 1:-1, 1:-1, 4]) / p.dy
         + (f[1:-1, 1:-1, 2:, 5] - f[1:-1, 1:-1, 1:-1, 5]) / p.dz)
    return d[3:-3, 3:-3, 3:-3]  # away from the zero ghost layers


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("g_prof", [True, False])
@pytest.mark.parametrize("wfac", [0.15, 0.3])
def test_longitudinal_terms_cancel_the_divergence(ndim, g_prof, wfac):
    """The O(sigma) Ex (and Bx in 3D) terms of get_laser_fields_lp are the
    paraxial corrections that make the pulse divergence-free to first order
    in eps = 1/(om0 w0): without them max|div E| (max|div B|) of the sampled
    pulse is that of the transverse profile alone; with them it falls below
    2 eps of it (measured 0.5 to 1.4 eps over w0 = 1.2 to 2.9 um); a wrong
    sign or a missing factor of the terms would leave 0.5 to 2 of it."""
    p = small_case(ndim, nx=96, ny=96, nz=96, cap=16)
    lx = p.nx * p.dx
    las = laser(2.0, LAM0, wfac * 48 * p.dy, 4 * LAM0, xc=0.5 * lx, xf=0.55 * lx, y0=0.1, z0=-0.2)
    a = lp_pulse(las, g_prof)
    eps = 1.0 / (a.om0 * a.wy)
    f = lp_fields(p, a)
    f0 = f.copy()
    f0[..., 0] = 0.0
    ratio = np.abs(_div_e(f, p)).max() / np.abs(_div_e(f0, p)).max()
    assert ratio < 2 * eps, (ratio, eps)
    if ndim == 3:
        f0 = f.copy()
        f0[..., 3] = 0.0
        ratio = np.abs(_div_b(f, p)).max() / np.abs(_div_b(f0, p)).max()
        assert ratio < 2 * eps, (ratio, eps)
