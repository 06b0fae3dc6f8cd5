"""PWFA bunch set-up on the device (agpu_beam_inject / agpu_beam_potential)
against the oracle and closed forms.

* Poisson solve (cuFFT DST-I of the odd extension) on pure sine modes: the
  reference solver's closed-form answer to 1e-12, on small grids and on the
  full 512x256x256 grid of the PWFA case.
* Poisson solve of a random density against the oracle's direct DST: 1e-12.
* beam_inject, FP64 form: the kept (in-box) records bit-exact, jc(1)
  (potential), jc(2) and the fields within 1e-11 of the oracle (the charge
  deposit sums with atomics, so only the summation order differs).
* beam_inject, FP32 split form: fields within 1e-6 of the oracle (one FP32
  rounding of the sum).
* After the set-up, the standard cycle (gather, push, deposit, Yee) with the
  bunch and a plasma, deterministic FP64 form: particles bit-exact against
  the oracle for 6 steps; the same for the reference's own PWFA route, the
  envelope cycle (particles, fields and env bit-exact).
* Linearity at the full PWFA size: fields(A u B) = fields(A) + fields(B).
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.beam import bunch_records
from aladyn_b200.config import Grid, make_params
from aladyn_b200.sim import PicDevice
from oracle.oracle import Oracle
from tests.helpers import grid_pwfa, inside_box, plasma_source, pwfa_bunch, sine_mode, sine_mode_potential

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ndim,dims,mode", [
    (3, (40, 24, 20), (3, 5, 2)),
    (3, (40, 24, 20), (39, 0, 19)),
    (2, (64, 32, 1), (0, 7, 0)),
    (3, (512, 256, 256), (6, 11, 4)),
])
def test_poisson_pure_modes(ndim, dims, mode):
    g = Grid(ndim, dims[0], dims[1], dims[2], k0=5.0, yx_rat=2.5, zx_rat=2.5, cfl=0.8)
    p = make_params(g, capacity=(16, 0, 0, 0))
    dev = PicDevice(p)
    rho = sine_mode(p, dev.n1p, dev.n2p, dev.n3p, *mode)
    gam2 = 1957.0 ** 2
    pot = dev.beam_potential(rho, gam2)
    expect = sine_mode_potential(p, rho, *mode, gam2)
    assert np.abs(pot - expect).max() <= 1e-12 * np.abs(expect).max()


@pytest.mark.parametrize("ndim", [2, 3])
def test_poisson_random_density_matches_oracle(ndim):
    p = make_params(grid_pwfa(ndim, 40, 24, 18), capacity=(16, 0, 0, 0))
    dev, ora = PicDevice(p), Oracle(p)
    rng = np.random.default_rng(5)
    rho = np.asfortranarray(rng.standard_normal((dev.n1p, dev.n2p, dev.n3p)))
    a = dev.beam_potential(rho, 25.0)
    b = ora.beam_potential(rho, 25.0)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    interior = np.zeros_like(rho, dtype=bool)
    k = slice(2, 2 + p.nz) if ndim == 3 else slice(0, 1)
    interior[2:2 + p.nx, 2:2 + p.ny, k] = True
    assert np.array_equal(a[~interior], rho[~interior])  # ghosts pass through


def _inject_pair(ndim, precision, nb=20000):
    p = make_params(grid_pwfa(ndim), precision=precision, capacity=(200_000, 0, 0, 0))
    dev = PicDevice(p)
    ora = Oracle(make_params(grid_pwfa(ndim), precision=AGPU_FP64, capacity=(200_000, 0, 0, 0)))
    b = pwfa_bunch(p, nb=nb)
    rec = bunch_records(p, b, n0_ref=0.1)
    zero = np.zeros(dev.field_shape(), order="F")
    dev.set_fields(zero)
    ora.set_fields(zero)
    assert dev.beam_inject(0, rec, b.gam) == 0
    assert ora.beam_inject(0, rec, b.gam) == 0
    return p, dev, ora, rec


@pytest.mark.parametrize("ndim", [2, 3])
def test_beam_inject_fp64_matches_oracle(ndim):
    p, dev, ora, rec = _inject_pair(ndim, AGPU_FP64)
    kept = inside_box(p, rec)
    assert 0 < kept.shape[0] < rec.shape[0]  # the box cuts the bunch tails
    assert dev.count(0) == ora.count(0) == kept.shape[0]
    got = dev.get_species(0)
    assert np.array_equal(got.view(np.uint64), ora.get_species(0).view(np.uint64))
    fa, fb = dev.get_fields(), ora.get_fields()
    for c in range(p.nfield):
        scale = max(np.abs(fb[..., c]).max(), 1e-300)
        assert np.abs(fa[..., c] - fb[..., c]).max() <= 1e-11 * scale, c
    # agpu_get_currents returns djc(c) * jc, as the reference's curr_mpi_collect
    # scales it; the oracle returns the raw array
    ja, jb = dev.get_currents(), ora.get_currents()
    for c in range(2):
        ref = p.djc[c] * jb[..., c]
        assert np.abs(ja[..., c] - ref).max() <= 1e-11 * np.abs(ref).max(), c


@pytest.mark.parametrize("ndim", [2, 3])
def test_beam_inject_fp32_split_matches_oracle(ndim):
    p, dev, ora, rec = _inject_pair(ndim, AGPU_FP32_SPLIT)
    kept = inside_box(p, rec)
    assert dev.count(0) == kept.shape[0]
    fa, fb = dev.get_fields(), ora.get_fields()
    for c in range(p.nfield):
        scale = max(np.abs(fb[..., c]).max(), 1e-300)
        assert np.abs(fa[..., c] - fb[..., c]).max() <= 1e-6 * scale, c
    back = dev.get_species(0)
    assert np.abs(back[:, 0] - kept[:, 0]).max() < 1e-5 * p.dx * p.nx


def test_pwfa_cycle_after_setup_bitexact():
    """The PWFA pairing on a small grid: plasma + bunch, standard cycle, FP64."""
    kw = dict(capacity=(400_000, 0, 0, 0), w_sh=4)
    p = make_params(grid_pwfa(3, 48, 24, 24), **kw)
    dev, ora = PicDevice(p), Oracle(make_params(grid_pwfa(3, 48, 24, 24), **kw))
    src = plasma_source(p, ic=0, npx=1, npy=1, npz=1, x_start_frac=0.1, n_over_n0=1.0)
    b = pwfa_bunch(p, nb=5000, sxb=1.5, syb=1.0)
    rec = bunch_records(p, b, n0_ref=0.1)
    zero = np.zeros(dev.field_shape(), order="F")
    for s in (dev, ora):
        s.set_fields(zero)
        s.set_plasma_source(src)
        s.load_plasma(0)
    assert dev.beam_inject(0, rec, b.gam) == 0
    assert ora.beam_inject(0, rec, b.gam) == 0
    fa, fb = dev.get_fields(), ora.get_fields()
    assert np.abs(fa - fb).max() <= 1e-11 * np.abs(fb).max()
    # restart both from identical fields so the cycle comparison is bit-exact
    dev.set_fields(fb)
    dev.set_deterministic(True)
    t = 0.0
    for it in range(6):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        assert out.np[0] == oo.np[0]
        t += p.dt
    a, c = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), c.view(np.uint64))
    fa, fb = dev.get_fields(), ora.get_fields()
    assert np.abs(fa - fb).max() <= 1e-12 * np.abs(fb).max()


def test_beam_inject_linearity_full_pwfa_grid():
    """512x256x256 (dx 0.2 um, dy = dz 0.5 um): the set-up is linear in the
    bunch: fields(A u B) = fields(A) + fields(B) to round-off."""
    g = Grid(3, 512, 256, 256, k0=5.0, yx_rat=2.5, zx_rat=2.5, cfl=0.8)
    p = make_params(g, capacity=(2_000_000, 0, 0, 0))
    ba = pwfa_bunch(p, nb=400_000, sxb=5.0, syb=3.0, seed=1)
    bb = pwfa_bunch(p, nb=400_000, sxb=5.0, syb=3.0, seed=2)
    ra, rb = bunch_records(p, ba, 0.1), bunch_records(p, bb, 0.1)
    fields = []
    for rec in (ra, rb, np.concatenate([ra, rb], axis=0)):
        dev = PicDevice(p)
        dev.set_fields(np.zeros(dev.field_shape(), order="F"))
        assert dev.beam_inject(0, rec, ba.gam) == 0
        f = dev.get_fields()
        fields.append(f[..., [1, 2, 4, 5]])  # Ey, Ez, By, Bz
        dev.close()
    fa, fb, fab = fields
    assert np.isfinite(fab).all()
    assert np.abs(fab - fa - fb).max() <= 1e-11 * np.abs(fab).max()


def test_pwfa_envelope_route_after_setup_bitexact():
    """The reference's own PWFA route (Env_cycle: beam_inject, then env_run
    every step, a0 = 0) on a small grid: plasma + bunch in species 0, the
    envelope cycle, FP64 deterministic mode: particles, fields and env
    bit-exact against the oracle for 6 steps."""
    from aladyn_b200.config import env_params
    kw = dict(capacity=(400_000, 0, 0, 0), w_sh=4)
    g = grid_pwfa(3, 48, 24, 24)
    p = make_params(g, **kw)
    dev, ora = PicDevice(p), Oracle(make_params(g, **kw))
    ep = env_params(g, 0.8, 2)
    dev.env_enable(ep)
    ora.env_enable(ep)
    src = plasma_source(p, ic=0, npx=1, npy=1, npz=1, x_start_frac=0.1, n_over_n0=1.0)
    b = pwfa_bunch(p, nb=5000, sxb=1.5, syb=1.0)
    rec = bunch_records(p, b, n0_ref=0.1)
    zero = np.zeros(dev.field_shape(), order="F")
    for s in (dev, ora):
        s.set_fields(zero)
        s.set_plasma_source(src)
        s.load_plasma(0)
    assert dev.beam_inject(0, rec, b.gam) == 0
    assert ora.beam_inject(0, rec, b.gam) == 0
    dev.set_fields(ora.get_fields())
    dev.set_deterministic(True)
    for it in range(1, 7):
        t = it * p.dt
        out = dev.env_run(t, it)
        rc, oo = ora.env_run(t, it)
        assert rc == 0 and out.error_bits == 0
        assert out.np[0] == oo.np[0]
    a, c = dev.get_species(0), ora.get_species(0)
    assert np.array_equal(a.view(np.uint64), c.view(np.uint64))
    assert np.array_equal(dev.get_fields(), ora.get_fields())
    assert np.array_equal(dev.get_envelope(), ora.get_envelope())
