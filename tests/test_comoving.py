"""The comoving frame (w_speed < 0, vbeam = -w_speed; set_init_param.f90:
239-245) in the oracle: the x advection of the fields (field_xadvect,
src/fields/grid_fields.f90:210-324, with trid_der1 37-77) against the
formula and a dense tridiagonal solve, the particle shift x -= dt vbeam of
the pushers (boris_push.f90:161-166, 288-294), comoving_coordinate's
source shift, removal and injection (src/dynamics/window.f90:227-275), and
the reduced envelope solver env_lpf_solve with ib = 0
(grid_fields.f90:696-858) against a numpy restatement, bit for bit."""
import numpy as np
import pytest

from aladyn_b200.sim import pack_slot
from oracle.oracle import Oracle
from tests.helpers import plasma_source, small_case
from tests.test_envelope import env_case, numpy_env_bds, numpy_env_grad, numpy_init, pulse


def _interior(p):
    i1, i2, j1, j2 = 2, p.nx + 1, 2, p.ny + 1
    k1, k2 = (2, p.nz + 1) if p.ndim == 3 else (0, 0)
    return i1, i2, j1, j2, k1, k2


def _random_fields(p, o, seed=5):
    rng = np.random.default_rng(seed)
    ebf = np.asfortranarray(rng.standard_normal(o.field_shape()))
    o.set_fields(ebf)
    return ebf


@pytest.mark.parametrize("ndim", [2, 3])
def test_xadvect_explicit_matches_formula(ndim):
    p = small_case(ndim, nx=32, ny=12, nz=8)
    p.w_speed = -1.0
    o = Oracle(p)
    ebf = _random_fields(p, o)
    nc = 2 if ndim == 2 else 3
    dth, v = 0.5 * p.dt, -1.0
    o.field_xadvect(dth, v, 1, nc, 0)
    got = o.get_fields()
    i1, i2, j1, j2, k1, k2 = _interior(p)
    J, K = slice(j1, j2 + 1), slice(k1, k2 + 1)
    want = ebf.copy(order="F")
    aphx_exp = 0.5 * v * (dth * p.dx_inv)
    for c in range(nc):
        f = want[..., c]
        f[i1 - 1, J, K] = f[i1 + 1, J, K]
        f[i2 + 1, J, K] = f[i2, J, K]
        new = f[i1:i2 + 1, J, K] - aphx_exp * (f[i1 + 1:i2 + 2, J, K] - f[i1 - 1:i2, J, K])
        f[i1:i2 + 1, J, K] = new
    assert np.array_equal(got, want)


@pytest.mark.parametrize("ndim", [2, 3])
def test_xadvect_implicit_solves_the_tridiagonal_system(ndim):
    """isch = 2: each row u solves aphx_exp (u_{i+1} - u_{i-1}) + u_i = f_i on
    the inner rows with u_1 = f_1 and u_n = f_n (b1 = bn = 1, c1 = an = 0)."""
    p = small_case(ndim, nx=32, ny=12, nz=8)
    p.w_speed = -1.0
    o = Oracle(p)
    ebf = _random_fields(p, o, seed=9)
    nf = 3 if ndim == 2 else 6
    nc = 2 if ndim == 2 else 3
    dth, v = 0.5 * p.dt, -1.0
    o.field_xadvect(dth, v, nc + 1, nf, 2)
    got = o.get_fields()
    i1, i2, j1, j2, k1, k2 = _interior(p)
    n = i2 - i1 + 1
    ax = 0.5 * v * (dth * p.dx_inv)
    m = np.eye(n)
    for r in range(1, n - 1):
        m[r, r - 1] = -ax
        m[r, r + 1] = ax
    worst = 0.0
    for c in range(nc, nf):
        for k in range(k1, k2 + 1):
            for j in range(j1, j2 + 1):
                u = np.linalg.solve(m, ebf[i1:i2 + 1, j, k, c])
                worst = max(worst, np.abs(got[i1:i2 + 1, j, k, c] - u).max() / np.abs(u).max())
                assert got[i1 - 1, j, k, c] == ebf[i1 + 1, j, k, c]
                assert got[i2 + 1, j, k, c] == ebf[i2, j, k, c]
    assert worst < 1e-13, worst
    # the E components are untouched
    assert np.array_equal(got[..., :nc], ebf[..., :nc])


@pytest.mark.parametrize("ndim", [2, 3])
def test_particles_at_rest_drift_by_minus_vbeam_dt(ndim):
    """Zero fields and weightless particles at rest: every step moves x by
    exactly -dt vbeam (x - dt vbeam in FP64), y and z stay, fields stay 0."""
    p = small_case(ndim, nx=48, ny=16, nz=12, cap=1000, w_sh=1000)
    vb = 0.95
    p.w_speed = -vb
    o = Oracle(p)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    rng = np.random.default_rng(2)
    n = 40
    rec = np.zeros((n, 7 if ndim == 3 else 5), order="F")
    rec[:, 0] = rng.uniform(p.xmn + 30 * p.dx, p.xmn + 40 * p.dx, n)
    rec[:, 1] = rng.uniform(p.ymn + 4 * p.dy, p.ymn + 10 * p.dy, n)
    if ndim == 3:
        rec[:, 2] = rng.uniform(p.zmn + 4 * p.dz, p.zmn + 8 * p.dz, n)
    rec[:, -1] = pack_slot(-1, 0, 0.0)
    o.set_species(0, rec)
    x = rec[:, 0].copy()
    for it in range(1, 11):
        rc, out = o.lp_run(it * p.dt, it)
        assert rc == 0
        x = x - p.dt * vb
    got = o.get_species(0)
    assert np.array_equal(got[:, 0], x)
    assert np.array_equal(got[:, 1:ndim], rec[:, 1:ndim])
    assert not o.get_fields().any()


@pytest.mark.parametrize("ndim", [2, 3])
def test_comoving_coordinate_injects_the_moving_target(ndim):
    """Every w_sh steps the plasma source moves left by vbeam w_sh dt: the
    lattice columns that cross xmax are injected, particles stay inside
    (gxmin, gxmax], and the counts add up."""
    p = small_case(ndim, nx=48, ny=16, nz=12, w_sh=4)
    p.w_speed = -1.0
    o = Oracle(p)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    src = plasma_source(p, x_start_frac=0.85)
    o.set_plasma_source(src)
    o.load_plasma(0)
    n = o.count(0)
    injected = 0
    for it in range(1, 17):
        rc, out = o.lp_run(it * p.dt, it)
        assert rc == 0
        assert out.np[0] == n - out.removed[0] + out.injected[0]
        if it % 4 != 0:
            assert out.injected[0] == 0
        n = out.np[0]
        injected += out.injected[0]
    assert injected > 0
    part = o.get_species(0)
    assert (part[:, 0] > p.gxmin).all() and (part[:, 0] <= p.gxmax).all()
    # the source started at 85% of the box and moved 16 dt to the left
    assert part[:, 0].min() < p.gxmin + 0.85 * p.nx * p.dx - 8 * p.dt


def numpy_comoving_vacuum_step(p, ep, env):
    """One env_run of an empty box in the comoving frame: env_bds, the source
    -ompe * 0 * A plus the transverse Laplacian, -dt on the row jy1 only,
    first_der's rotation, the three-point inversion, the update,
    env_fields_average and env_grad.  Returns (env, av)."""
    E = env.copy(order="F")
    numpy_env_bds(p, E)
    i1, i2, j1, j2, k1, k2 = _interior(p)
    X, Y, Z = slice(i1, i2 + 1), slice(j1, j2 + 1), slice(k1, k2 + 1)

    def sh(a, di=0, dj=0, dk=0):
        return a[i1 + di:i2 + 1 + di, j1 + dj:j2 + 1 + dj, k1 + dk:k2 + 1 + dk]

    om0, dt = ep.om0, p.dt
    dy2, dz2 = p.dy_inv * p.dy_inv, p.dz_inv * p.dz_inv
    A = np.zeros(E.shape[:3] + (2,), order="F")   # av(1:2); their x ghosts stay 0
    for q in range(2):
        e = E[..., q]
        a = -p.ompe * np.zeros_like(sh(e)) * sh(e)
        a = a + dy2 * ((sh(e, 0, 1) - sh(e)) - (sh(e) - sh(e, 0, -1)))
        if p.ndim == 3:
            a = a + dz2 * ((sh(e, 0, 0, 1) - sh(e)) - (sh(e) - sh(e, 0, 0, -1)))
        A[X, Y, Z, q] = a
    A[X, j1, Z, :] = -dt * A[X, j1, Z, :]
    dx1_inv = 0.5 * p.dx_inv
    a1, a2 = A[..., 0], A[..., 1]
    w1 = om0 * sh(a2) + dx1_inv * (sh(a1, 1) - sh(a1, -1))
    w2 = -om0 * sh(a1) + dx1_inv * (sh(a2, 1) - sh(a2, -1))
    A[X, Y, Z, 0] = w1
    A[X, Y, Z, 1] = w2
    dx_norm = p.dx_inv / om0
    dx2_norm = dx_norm * dx_norm
    for q in range(2):
        a = A[..., q]
        w = dx2_norm * (sh(a, 1) - 2. * sh(a) + sh(a, -1))
        A[X, Y, Z, q] = (sh(a) - w) / (om0 * om0)
    for q in range(2):
        v = A[X, Y, Z, q] + E[X, Y, Z, q + 2]
        E[X, Y, Z, q + 2] = E[X, Y, Z, q]
        E[X, Y, Z, q] = v
    av = np.zeros(E.shape[:3] + (p.ndim + 1,), order="F")
    s1, s2 = E[X, Y, Z, 0] + E[X, Y, Z, 2], E[X, Y, Z, 1] + E[X, Y, Z, 3]
    av[X, Y, Z, 0] = (1.0 / 8.) * (s1 * s1 + s2 * s2)
    numpy_env_grad(p, av)
    return E, av


@pytest.mark.parametrize("ndim", [2, 3])
def test_comoving_envelope_vacuum_step_matches_numpy(ndim):
    p, g, ep = env_case(ndim)
    p.w_speed = -1.0
    o = Oracle(p)
    o.env_enable(ep)
    env0 = numpy_init(p, pulse(p))
    o.set_envelope(env0)
    rc, _ = o.env_run(p.dt, 1)
    assert rc == 0
    want_env, want_av = numpy_comoving_vacuum_step(p, ep, env0)
    assert np.array_equal(o.get_envelope(), want_env)
    assert np.array_equal(o.get_env_source(), want_av)
