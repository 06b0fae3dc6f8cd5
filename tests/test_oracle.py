"""CPU checks of the oracle: published known-answer vectors and the method's
invariants (the reference ships no golden vectors of its own)."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle.oracle import Oracle, build_ionization_table, load
from tests.helpers import laser_fields, plasma_source, small_case


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_philox_known_answers():
    """Random123's published Philox4x32-10 vectors."""
    lib = load()
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        c = (C.c_uint32 * 4)(*ctr)
        o = (C.c_uint32 * 4)()
        lib.ora_philox(c, key[0], key[1], o)
        assert tuple(o) == want


def test_shapes_partition_of_unity():
    lib = load()
    rng = np.random.default_rng(3)
    ax, axh = (C.c_double * 3)(), (C.c_double * 3)()
    ix, ih = C.c_int(), C.c_int()
    for x in rng.uniform(0.0, 50.0, 2000):
        lib.ora_shape_qlh(x, ax, axh, C.byref(ix))
        assert abs(sum(ax) - 1.0) < 1e-15 and abs(axh[0] + axh[1] - 1.0) < 1e-15
        assert min(ax) >= 0.0 and min(axh[0], axh[1]) >= 0.0
        # quadratic weights on nodes ix..ix+2 reproduce the position (first moment)
        xx = 3.0 + x
        m = sum(ax[q] * (ix.value + q) for q in range(3))
        assert abs(m - xx) < 1e-12
        lib.ora_shape_qqh(x, ax, axh, C.byref(ix), C.byref(ih))
        assert abs(sum(ax) - 1.0) < 1e-15 and abs(sum(axh) - 1.0) < 1e-15
        lib.ora_shape_qden(x, ax, C.byref(ix))
        assert abs(sum(ax) - 1.0) < 1e-15


@pytest.mark.parametrize("ndim,shape", [(2, 0), (3, 0), (2, 1), (3, 1)])
def test_esirkepov_discrete_continuity(ndim, shape):
    """rho^1 - rho^0 + c * (J(i) - J(i-1)) summed over axes = 0 at round-off,
    c = 1/2 in 2D and 1/3 in 3D (the djc normalisation,
    src/start/set_init_param.f90:92-103); quadratic (the reference) and the
    cubic extension, each with its own density."""
    p = small_case(ndim, nx=16, ny=16, nz=16, cap=10)
    p.shape = shape
    o = Oracle(p)
    rng = np.random.default_rng(7 + ndim)
    shape = (o.n1p, o.n2p, o.n3p)
    cfac = 0.5 if ndim == 2 else 1.0 / 3.0
    for _ in range(100):
        x0 = rng.uniform(3.0, 12.0, ndim)
        x1 = x0 + rng.uniform(-0.95, 0.95, ndim)
        w = np.float32(rng.uniform(-2, 2))
        o.lib.ora_zero_currents(o.h)
        o.lib.ora_deposit_move(o.h, _dp(x1), _dp(x0), C.c_float(w))
        jc = o.get_currents()
        r0 = np.zeros(shape, order="F")
        r1 = np.zeros(shape, order="F")
        o.lib.ora_rho_one(o.h, _dp(r0), _dp(x0), float(w))
        o.lib.ora_rho_one(o.h, _dp(r1), _dp(x1), float(w))
        div = sum(jc[..., a] - np.roll(jc[..., a], 1, axis=a) for a in range(ndim))
        res = (r1 - r0) + cfac * div
        assert np.abs(res).max() < 1e-14 * max(1.0, abs(float(w)))


def test_cubic_shapes_partition_of_unity_and_symmetry():
    """Cubic B-spline weights (the cden weights) and the quadratic half-node
    weights sum to one; the cubic weights are the B-spline of the distance
    to each node, so mirroring the offset mirrors the weights."""
    lib = load()
    a4 = (C.c_double * 4)()
    ah = (C.c_double * 3)()
    ix, ih = C.c_int(), C.c_int()
    for x in np.linspace(0.0, 9.999, 401):
        lib.ora_shape_cubic(float(x), a4, ah, C.byref(ix), C.byref(ih))
        assert abs(sum(a4) - 1.0) < 1e-15 and abs(sum(ah) - 1.0) < 1e-15
        s = 3.0 + x - ix.value
        bs = lambda d: (2 - abs(d)) ** 3 / 6 if abs(d) >= 1 else 2 / 3 - d * d + abs(d) ** 3 / 2
        for q in range(4):
            assert abs(a4[q] - bs(s + 1 - q)) < 1e-14


def test_boris_pure_magnetic_field_conserves_momentum():
    """Exact-gamma Boris (boris_push.f90:124-152) in a uniform Bz with zero
    current: |p| is conserved to round-off."""
    p = small_case(3, nx=64, ny=32, nz=32, cap=16, w_sh=0)
    o = Oracle(p)
    ebf = np.zeros(o.field_shape(), order="F")
    ebf[..., 5] = 3.0
    o.set_fields(ebf)
    part = np.zeros((1, 7), order="F")
    part[0, 0] = 0.5 * p.nx * p.dx
    part[0, 1] = 0.0
    part[0, 2] = 0.0
    part[0, 3:6] = [0.3, 0.2, 0.05]
    from aladyn_b200.sim import pack_slot
    part[0, 6] = pack_slot(-1, 0, 0.0)  # zero weight: no current
    o.set_species(0, part)
    p0 = np.linalg.norm(part[0, 3:6])
    t = 0.0
    for it in range(1, 16):  # before the open-boundary disturbance reaches it
        rc, out = o.lp_run(t, it)
        assert rc == 0
        t += p.dt
    q = o.get_species(0)
    assert q.shape[0] == 1
    assert abs(np.linalg.norm(q[0, 3:6]) - p0) < 1e-13 * p0


def test_vacuum_yee_pulse_stays_bounded():
    """A vacuum laser pulse under the leapfrog Yee update with the Mur-type
    open boundaries stays bounded at CFL 0.8: the field energy never grows
    (the open boundaries only absorb) and most of it stays in the box."""
    p = small_case(2, nx=96, ny=48, cap=16, w_sh=0)
    o = Oracle(p)
    o.set_fields(laser_fields(p, a0=1.0))

    def energy(f):
        return float(np.sum(f[2:p.nx + 2, 2:p.ny + 2, 0, :] ** 2))

    e0 = energy(o.get_fields())
    t = 0.0
    for it in range(30):
        o.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    e1 = energy(o.get_fields())
    assert np.isfinite(e1) and 0.5 * e0 < e1 <= 1.001 * e0


def test_ionization_table_matches_closed_form_adk():
    """One-level ADK (model 1): w = 1 - exp(-dt_fs * omega_a * W_ADK(E)) with
    W_ADK = C_n* (2 V^(3/2)/E)^(2n*-1) exp(-2 V^(3/2)/(3E)) for nitrogen's first
    level (ionize.f90:59-72, 174-187; ionz_data.f90:187-245, 776-803)."""
    dt, e_max = 0.03, 3.0
    tab, de_inv = build_ionization_table(7, 0, 1, e_max, dt)
    v_h, euler, pig = 13.5984, 2.71828, 3.141592653589793
    v = 14.53 / v_h
    nstar = 1.0 / math.sqrt(v)
    vfact = v * math.sqrt(v)
    cn = (2 * euler / nstar) ** (2 * nstar) * 3 / (2 * pig * nstar) * 0.5 * v
    dt_fs = 10 * dt / 3
    for i in (500, 2000, 5000, 9999):
        e = (e_max / 10000) * i
        f2 = 2 * vfact / e
        w = cn * f2 ** (2 * nstar - 1) * math.exp(-f2 / 3)
        w = 0.0 if w < 1e-10 else w
        want = 1 - math.exp(-dt_fs * 41.3 * w)
        assert abs(tab[i, 0] - want) <= 1e-12 * max(want, 1e-300)
    assert abs(de_inv - 10000 / e_max) < 1e-9
    assert np.all(tab[:, 7] == 0.0)  # fully ionized row


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_lwfa_steps_with_window(ndim):
    """A short LWFA run: the window shifts by nint(dx_inv * xlapse) cells,
    particles are injected and removed, no error bits."""
    p = small_case(ndim, nx=48, ny=24, nz=12, cap=200_000)
    o = Oracle(p)
    o.set_fields(laser_fields(p))
    o.set_plasma_source(plasma_source(p, x_start_frac=0.0))
    o.load_plasma(0)
    t, shifts, xl = 0.0, 0, 0.0
    for it in range(21):
        rc, out = o.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        if it % p.w_sh == 0 and it > 0:
            xl += p.w_speed * p.dt * p.w_sh
            assert out.nshx == int(math.floor(p.dx_inv * xl + 0.5)) - shifts
            shifts += out.nshx
            assert out.injected[0] > 0 and out.removed[0] > 0
        t += p.dt
    assert abs(o.xmn() - shifts * p.dx) < 1e-12


def test_threaded_oracle_matches_serial():
    """The threaded CPU baseline (per-thread current copies) agrees with the
    serial oracle to round-off."""
    p = small_case(3, nx=32, ny=16, nz=16, cap=100_000)
    outs = []
    for th in (1, 4):
        o = Oracle(small_case(3, nx=32, ny=16, nz=16, cap=100_000), threads=th)
        o.set_fields(laser_fields(p))
        o.set_plasma_source(plasma_source(p))
        o.load_plasma(0)
        t = 0.0
        for it in range(3):
            o.lp_run(t, it, initial_time=(it == 0))
            t += p.dt
        outs.append(o.get_fields())
    a, b = outs
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_empty_species_with_window(ndim):
    """No particles at all: the step, the window shift (no injection source)
    and the field update run, nothing is counted and no error bit is set."""
    p = small_case(ndim, nx=40, ny=20, nz=12, cap=1000)
    o = Oracle(p)
    o.set_fields(laser_fields(p))
    e0 = float(np.sum(o.get_fields() ** 2))
    t = 0.0
    for it in range(12):
        rc, out = o.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        assert out.np[0] == 0 and out.injected[0] == 0 and out.removed[0] == 0
        t += p.dt
    e1 = float(np.sum(o.get_fields() ** 2))
    assert np.isfinite(e1) and e1 <= 1.5 * e0
    assert o.count(0) == 0


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_box_edge_removal(ndim):
    """reset_all_part_dist keeps xl < x <= xr per axis (mpi_part_interface.f90:
    467-523): at rest in zero fields, a record exactly on the right box edge
    stays, one just beyond it and one exactly on the left edge leave."""
    from aladyn_b200.sim import pack_slot
    p = small_case(ndim, nx=40, ny=20, nz=12, cap=1000)
    o = Oracle(p)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    yc = 0.5 * (p.gymin + p.gymax)
    zc = 0.5 * (p.gzmin + p.gzmax)
    xs = [p.gxmax, p.gxmax + 1e-9 * p.dx, p.gxmin, 0.5 * (p.gxmin + p.gxmax)]
    rec = np.zeros((len(xs), 2 * ndim + 1))
    rec[:, 0] = xs
    rec[:, 1] = yc
    if ndim == 3:
        rec[:, 2] = zc
    rec[:, -1] = pack_slot(-1, 0, 1.0)
    o.set_species(0, rec)
    rc, out = o.lp_run(0.0, 1)  # no window shift on iteration 1
    assert rc == 0 and out.error_bits == 0
    kept = o.get_species(0)
    assert kept.shape[0] == 2
    assert sorted(kept[:, 0].tolist()) == sorted([p.gxmax, xs[3]])
