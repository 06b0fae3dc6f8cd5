"""Known answers for the oracle's particle push (lpf_momenta_and_positions,
src/dynamics/boris_push.f90:75-168): the momentum at the half step is the
solution p^n of the implicit equation

    p^n = p^{n-1/2} + a q E + (p^n / gamma(p^n)) x (a q B),  a = dt / (2 m),

and p^{n+1/2} = 2 p^n - p^{n-1/2}; then x += dt p^{n+1/2} / gamma.  Three
exact consequences, each checked on a test particle of zero weight (no
current) in uniform fields, before the open boundaries' disturbance can
reach it, in 2D and 3D:

* crossed fields E = E0 y, B = B0 z: a particle moving at the drift
  velocity v = E0 / B0 along x (relativistic here, gamma = 2.29) feels no
  force, so its momentum stays exactly p and x advances by v dt a step;
* B = B0 z alone: p^{n+1/2} is p^{n-1/2} rotated by theta with
  tan(theta / 2) = |a q B| / gamma(p^n) and |p^n| = |p| cos(theta / 2), so
  cos^2(theta / 2) solves P^2 c^4 + (1 + b^2 - P^2) c^2 - 1 = 0;
* E = E0 x alone: p grows by q E0 dt / m every step, and x by the sum of
  dt p / gamma."""
import math

import numpy as np
import pytest

from aladyn_b200.sim import pack_slot
from oracle.oracle import Oracle
from tests.helpers import small_case


def _run(ndim, fields, p_init, steps):
    p = small_case(ndim, nx=64, ny=32, nz=32, cap=16, w_sh=0)
    o = Oracle(p)
    ebf = np.zeros(o.field_shape(), order="F")
    for comp, val in fields.items():
        ebf[..., comp] = val
    o.set_fields(ebf)
    nd = 2 * ndim + 1
    part = np.zeros((1, nd), order="F")
    part[0, 0] = 0.4 * p.nx * p.dx
    part[0, ndim:2 * ndim] = p_init[:ndim]
    part[0, -1] = pack_slot(-1, 0, 0.0)  # an electron of zero weight
    o.set_species(0, part)
    hist = [part[0].copy()]
    t = 0.0
    for it in range(1, steps + 1):
        rc, _ = o.lp_run(t, it)
        assert rc == 0
        q = o.get_species(0)
        assert q.shape[0] == 1
        hist.append(q[0].copy())
        t += p.dt
    return p, np.array(hist)


def _comps(ndim):
    """(Ex, Ey, Bz) field indices."""
    return (0, 1, 2) if ndim == 2 else (0, 1, 5)


@pytest.mark.parametrize("ndim", [2, 3])
def test_drift_velocity_particle_moves_uniformly(ndim):
    ex, ey, bz = _comps(ndim)
    e0, b0 = 2.7, 3.0
    v = e0 / b0
    gam = 1.0 / math.sqrt(1.0 - v * v)
    p, h = _run(ndim, {ey: e0, bz: b0}, [gam * v, 0.0, 0.0], 12)
    assert gam > 2.2
    mom = h[:, ndim:2 * ndim]
    assert np.abs(mom[:, 0] - gam * v).max() <= 2e-15 * gam * v
    assert np.abs(mom[:, 1:]).max() <= 1e-14
    dx = np.diff(h[:, 0])
    assert np.abs(dx - p.dt * v).max() <= 1e-14 * p.dt


@pytest.mark.parametrize("ndim", [2, 3])
def test_rotation_angle_in_uniform_b(ndim):
    ex, ey, bz = _comps(ndim)
    b0 = 40.0
    p0 = np.array([0.6, -0.8, 0.0]) * 1.5
    steps = 12
    p, h = _run(ndim, {bz: b0}, p0, steps)
    big_p = np.linalg.norm(p0)
    b = 0.5 * p.dt * b0  # |a q B| for an electron of mass 1
    c2 = (-(1 + b * b - big_p ** 2) + math.sqrt((1 + b * b - big_p ** 2) ** 2 + 4 * big_p ** 2)) / (2 * big_p ** 2)
    theta = 2.0 * math.acos(math.sqrt(c2))
    # the same angle from tan(theta/2) = b / gamma(p^n), |p^n| = P cos(theta/2)
    assert abs(math.tan(theta / 2) - b / math.sqrt(1 + big_p ** 2 * c2)) < 1e-14
    mom = h[:, ndim:ndim + 2]
    ang = np.unwrap(np.arctan2(mom[:, 1], mom[:, 0]))
    step = np.diff(ang)
    # an electron (q = -1) in +Bz turns counter-clockwise in (px, py)
    assert np.abs(step - theta).max() <= 1e-13
    assert theta * steps > 1.0
    assert np.abs(np.linalg.norm(mom, axis=1) - big_p).max() <= 1e-14 * big_p


@pytest.mark.parametrize("ndim", [2, 3])
def test_uniform_e_acceleration(ndim):
    ex, ey, bz = _comps(ndim)
    e0 = 3.0
    steps = 15
    p, h = _run(ndim, {ex: e0}, [0.1, 0.0, 0.0], steps)
    k = np.arange(steps + 1)
    px = 0.1 - k * p.dt * e0  # q = -1, m = 1
    assert np.abs(h[:, ndim] - px).max() <= 1e-14
    dx = p.dt * px[1:] / np.sqrt(1.0 + px[1:] ** 2)
    assert np.abs(np.diff(h[:, 0]) - dx).max() <= 1e-14 * p.dt
    assert px[-1] < -1.0  # relativistic by the end
