"""A known answer for the oracle's field gather (set_part2d_hcell_acc /
set_part3d_hcell_acc, src/particles/grid_part_connect.f90:89-285): the
quadratic integer-node weights and the linear half-node weights both have
first moment equal to the particle's position, so a field that is linear
in x, y (and z) is gathered exactly, at its own staggered nodes

    Ex(i+1/2, j, k)  Ey(i, j+1/2, k)  Ez(i, j, k+1/2)
    Bx(i, j+1/2, k+1/2)  By(i+1/2, j, k+1/2)  Bz(i+1/2, j+1/2, k)

(node i at x = xmn + (i - 3) dx, 1-based with two ghost layers).  The
gathered values are read back through the push (boris_push.f90:75-168):
from rest with B = 0, p^{n+1/2} = dt q E / m; with E = 0 and the momentum
at right angles to the one B component that is set, the implicit
midpoint rotation gives d = s x b with d = p^{n+1/2} - p^{n-1/2},
s = (p^{n+1/2} + p^{n-1/2}) / gamma(p^n), b = (dt / 2) q B / m, so
b = -(s x d) / |s|^2 along that component.  A half-cell error in any
component's stagger would show as slope * dx / 2.  The cubic extension
(shape 1: cubic integer-node, quadratic half-node weights) has the same
first moments and gathers linear fields exactly too."""
import math

import numpy as np
import pytest

from aladyn_b200.sim import pack_slot
from oracle.oracle import Oracle
from tests.helpers import small_case

# (component index, axes staggered by half a cell) in the field array
STAGGER3 = {0: (0,), 1: (1,), 2: (2,), 3: (1, 2), 4: (0, 2), 5: (0, 1)}
STAGGER2 = {0: (0,), 1: (1,), 2: (0, 1)}


def _linear(p, comp, stagger, coef, shape):
    """coef[0] + sum_a coef[a + 1] * (coordinate a of the component's nodes)."""
    n1p, n2p, n3p = shape[:3]
    axes = []
    for a, (n, d, mn) in enumerate(zip((n1p, n2p, n3p), (p.dx, p.dy, p.dz), (p.xmn, p.ymn, p.zmn))):
        if a == 2 and p.ndim == 2:
            axes.append(np.zeros(1))
            continue
        off = 0.5 if a in stagger else 0.0
        axes.append(mn + (np.arange(1, n + 1) - 3 + off) * d)
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return coef[0] + coef[1] * X + coef[2] * Y + (coef[3] * Z if p.ndim == 3 else 0.0)


def _particles(p, n, rng, mom):
    nd = 2 * p.ndim + 1
    rec = np.zeros((n, nd), order="F")
    rec[:, 0] = rng.uniform(p.xmn + 8 * p.dx, p.xmn + (p.nx - 8) * p.dx, n)
    rec[:, 1] = rng.uniform(p.ymn + 6 * p.dy, p.ymn + (p.ny - 6) * p.dy, n)
    if p.ndim == 3:
        rec[:, 2] = rng.uniform(p.zmn + 6 * p.dz, p.zmn + (p.nz - 6) * p.dz, n)
    rec[:, p.ndim:2 * p.ndim] = mom
    rec[:, -1] = pack_slot(-1, 0, 0.0)  # electrons of zero weight
    return rec


def _one_step(p, fields, rec):
    o = Oracle(p)
    o.set_fields(fields)
    o.set_species(0, rec)
    rc, _ = o.lp_run(0.0, 1)
    assert rc == 0
    out = o.get_species(0)
    assert out.shape == rec.shape
    return o, out


def _expected(p, coef, rec):
    x = [rec[:, a] for a in range(p.ndim)]
    return coef[0] + coef[1] * x[0] + coef[2] * x[1] + (coef[3] * x[2] if p.ndim == 3 else 0.0)


@pytest.mark.parametrize("shape", [0, 1])
@pytest.mark.parametrize("ndim", [2, 3])
def test_linear_electric_field_is_gathered_exactly(ndim, shape):
    p = small_case(ndim, nx=48, ny=32, nz=32, cap=4096, w_sh=0)
    p.shape = shape
    rng = np.random.default_rng(11)
    rec = _particles(p, 2000, rng, 0.0)
    o = Oracle(p)
    fshape = o.field_shape()
    f = np.zeros(fshape, order="F")
    coefs = {}
    stag = STAGGER3 if ndim == 3 else STAGGER2
    for c in range(ndim):
        coefs[c] = rng.uniform(-0.4, 0.4, 4)
        f[..., c] = _linear(p, c, stag[c], coefs[c], fshape)
    _, out = _one_step(p, f, rec)
    for c in range(ndim):
        got = -out[:, ndim + c] / p.dt  # p^{n+1/2} = dt q E / m, q = -1, m = 1
        want = _expected(p, coefs[c], rec)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), c


@pytest.mark.parametrize("shape", [0, 1])
@pytest.mark.parametrize("ndim,comp", [(2, 2), (3, 3), (3, 4), (3, 5)])
def test_linear_magnetic_field_is_gathered_exactly(ndim, comp, shape):
    p = small_case(ndim, nx=48, ny=32, nz=32, cap=4096, w_sh=0)
    p.shape = shape
    rng = np.random.default_rng(17 + comp)
    axis = comp - 3 if ndim == 3 else 2  # the field's direction (x, y, z)
    n = 2000
    mom = rng.normal(0.0, 0.8, (n, 3))
    mom[:, axis] = 0.0
    rec = _particles(p, n, rng, mom[:, :ndim])
    o = Oracle(p)
    fshape = o.field_shape()
    f = np.zeros(fshape, order="F")
    coef = np.array([3.0, *rng.uniform(-0.6, 0.6, 3)])
    stag = STAGGER3 if ndim == 3 else STAGGER2
    f[..., comp] = _linear(p, comp, stag[comp], coef, fshape)
    _, out = _one_step(p, f, rec)
    p0 = np.zeros((n, 3))
    p1 = np.zeros((n, 3))
    p0[:, :ndim] = rec[:, ndim:2 * ndim]
    p1[:, :ndim] = out[:, ndim:2 * ndim]
    d = p1 - p0
    pn = 0.5 * (p1 + p0)
    s = (p1 + p0) / np.sqrt(1.0 + (pn ** 2).sum(axis=1))[:, None]
    b = -np.cross(s, d) / (s ** 2).sum(axis=1)[:, None]
    got = b[:, axis] / (0.5 * p.dt * -1.0)  # b = (dt / 2) q B / m
    want = _expected(p, coef, rec)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
    # the other components of b vanish (no field along them)
    others = [a for a in range(3) if a != axis]
    assert np.abs(b[:, others]).max() <= 1e-13
