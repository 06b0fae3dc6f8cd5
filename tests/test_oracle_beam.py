"""The oracle's PWFA bunch set-up (beam_inject) against closed forms: the
sine-transform Poisson solve on pure modes (with the reference's wavenumbers
and its x-axis forward scale), the total deposited charge, the stencil
relations of initial_beam_fields, the box selection, and the host bunch
generator's moments."""
import math

import numpy as np
import pytest

from aladyn_b200.beam import bunch_parameters, bunch_records
from aladyn_b200.config import make_params
from aladyn_b200.sim import unpack_slot
from oracle.oracle import Oracle
from tests.helpers import grid_pwfa, inside_box, pwfa_bunch, sine_mode, sine_mode_potential


@pytest.mark.parametrize("ndim,mode", [(3, (2, 3, 1)), (3, (0, 0, 0)), (3, (20, 9, 13)), (2, (0, 4, 0))])
def test_oracle_poisson_pure_modes(ndim, mode):
    p = make_params(grid_pwfa(ndim, 24, 16, 14), capacity=(10, 0, 0, 0))
    o = Oracle(p)
    rho = sine_mode(p, o.n1p, o.n2p, o.n3p, *mode)
    if ndim == 2:  # no x transform in 2D: any x profile passes through
        rho *= np.linspace(0.3, 1.7, o.n1p)[:, None, None]
    gam2 = 9.0
    pot = o.beam_potential(rho, gam2)
    expect = sine_mode_potential(p, rho, *mode, gam2)
    assert np.abs(pot - expect).max() <= 1e-13 * np.abs(expect).max()


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_grid_charge_total(ndim):
    p = make_params(grid_pwfa(ndim), capacity=(30000, 0, 0, 0))
    o = Oracle(p)
    rec = inside_box(p, bunch_records(p, pwfa_bunch(p, nb=3000), n0_ref=0.1))
    den = o.grid_charge(rec)
    q, _, w = unpack_slot(rec[:, -1])
    total = float((q.astype(np.float32) * w).astype(np.float64).sum())
    assert abs(den.sum() - total) <= 1e-10 * abs(total)


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_beam_fields_stencils(ndim):
    p = make_params(grid_pwfa(ndim), capacity=(30000, 0, 0, 0))
    o = Oracle(p)
    b = pwfa_bunch(p, nb=4000)
    rec = bunch_records(p, b, n0_ref=0.1)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    assert o.beam_inject(0, rec, b.gam) == 0
    f = o.get_fields()
    phi = o.get_currents()[..., 0]
    bet = math.sqrt(b.gam * b.gam - 1.) / b.gam
    I = slice(2, 2 + p.nx - 1)
    J = slice(2, 2 + p.ny)
    K = slice(2, 2 + p.nz) if ndim == 3 else slice(0, 1)
    ex = -p.dx_inv * (phi[3:3 + p.nx - 1, J, K] - phi[I, J, K]) / (b.gam * b.gam)
    assert np.allclose(f[I, J, K, 0], ex, rtol=0, atol=1e-14 * np.abs(ex).max())
    ey = f[..., 1]
    bz = 0.5 * bet * (ey[I, J, K] + ey[3:3 + p.nx - 1, J, K])
    assert np.allclose(f[I, J, K, p.nfield - 1], bz, rtol=0, atol=1e-14 * np.abs(bz).max())
    if ndim == 3:
        assert np.all(f[..., 3] == 0.0)
        ez = f[..., 2]
        by = -bet * (0.5 * (ez[I, J, K] + ez[3:3 + p.nx - 1, J, K]))
        assert np.allclose(f[I, J, K, 4], by, rtol=0, atol=1e-14 * np.abs(by).max())
    kept = inside_box(p, rec)
    assert 0 < kept.shape[0] < b.nb_tot  # the tails beyond the box are dropped
    assert o.count(0) == kept.shape[0]
    assert np.array_equal(o.get_species(0).view(np.uint64), kept.view(np.uint64))


def test_round_bunch_fields_are_transversely_symmetric():
    p = make_params(grid_pwfa(3, 48, 32, 32), capacity=(30000, 0, 0, 0))
    o = Oracle(p)
    b = pwfa_bunch(p, nb=20000, gam=100.0)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    assert o.beam_inject(0, bunch_records(p, b, n0_ref=0.1), b.gam) == 0
    f = o.get_fields()[2:50, 2:34, 2:34]
    ey, ez = np.abs(f[..., 1]).max(), np.abs(f[..., 2]).max()
    assert abs(ey / ez - 1.0) < 0.15
    assert np.abs(f[..., 0]).max() < 1e-2 * ey  # Ex ~ 1/gam^2


def test_bunch_generator_moments():
    p = make_params(grid_pwfa(3, 64, 32, 32), capacity=(10, 0, 0, 0))
    b = pwfa_bunch(p, nb=200000, sxb=3.0, syb=2.0, gam=1957.0)
    rec = bunch_records(p, b, n0_ref=0.1)
    prm = bunch_parameters(p, b, n0_ref=0.1)
    assert abs(rec[:, 0].mean() - b.xc) < 1e-9 and abs(rec[:, 1].mean()) < 1e-9 and abs(rec[:, 2].mean()) < 1e-9
    assert abs(rec[:, 3].mean() - b.gam) < 1e-6
    assert abs(rec[:, 0].std() / b.sxb - 1) < 0.01 and abs(rec[:, 1].std() / b.syb - 1) < 0.01
    assert abs(rec[:, 3].std() / (0.01 * b.dg * b.gam) - 1) < 0.01      # uniform spread of rms dg% gam
    assert abs(rec[:, 4].std() / (b.epsy / b.syb) - 1) < 0.01
    q, pi, w = unpack_slot(rec[:, -1])
    assert np.all(q == -1) and np.all(pi == 1) and np.all(w == np.float32(prm["jb_norm"]))
    vol = (2 * math.pi) ** 1.5 * b.sxb * b.syb ** 2
    assert abs(prm["rhob"] - 1e-6 * 200.0 / (1.6021766e-7 * vol) / 0.1) < 1e-9 * prm["rhob"]
