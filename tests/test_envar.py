"""Envar's reductions (src/diagnostics/diag_part_and_fields.f90:126-142,
172-220, 485-719) in the oracle's C restatement against a plain numpy
statement of the same formulas on the oracle's own records, 2D and 3D,
after a few laser-driven steps: the unweighted 3D momentum sums and the
weighted 2D ones, the angular momentum, the charge and energy sums,
max(gamma - 1), the momentum spreads, the 100-bin energy spectrum and the
field energies (dgvol = dx dy dy in 2D) and maxima; and the host's Envar
units (aladyn_b200.diagnostics.envar)."""
import numpy as np
import pytest

from aladyn_b200.diagnostics import ELECTRON_MASS, FIELD_ENERGY, MEV_TO_JOULE, envar, species_pmass
from aladyn_b200.sim import unpack_slot
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case


def _state(ndim, steps=6):
    p = small_case(ndim, nx=48, ny=24, nz=16, cap=200_000, w_sh=0)
    o = Oracle(p)
    o.set_fields(laser_fields(p, a0=3.0))
    o.set_plasma_source(plasma_source(p, x_start_frac=0.3))
    o.load_plasma(0)
    t = 0.0
    for it in range(steps):
        o.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    return p, o


def numpy_envar_species(p, part, pmass, ne=100):
    nd = int(p.ndim)
    ch, _, w = unpack_slot(part[:, -1])
    w64 = w.astype(np.float64)
    v = part[:, nd:2 * nd]
    gam = np.sqrt(1. + (v * v).sum(axis=1))
    g1 = gam - 1.
    ek = np.zeros(7)
    if nd == 3:
        ek[:3] = v.sum(axis=0)
        ek[3] = (w64 * (part[:, 1] * v[:, 2] - part[:, 2] * v[:, 1])).sum()
    else:
        ek[:2] = (w64[:, None] * v).sum(axis=0)
    ek[5] = (ch.astype(np.float32) * w).astype(np.float64).sum()
    ek[6] = (w64 * g1).sum()
    ekmax = g1.max()
    mean = ek[:nd] / part.shape[0]
    psig = np.zeros(3)
    psig[:nd] = ((v - mean) ** 2).sum(axis=0)
    ekem = pmass * ekmax
    nde = np.zeros(ne)
    if ekem >= 1e-6:
        xx = pmass * g1 / (ekem / ne)
        ix = np.minimum(np.floor(xx + 0.5).astype(int) + 1, ne)
        np.add.at(nde, ix - 1, w64)
    return ek, ekmax, psig, nde


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_envar_matches_numpy(ndim):
    p, o = _state(ndim)
    part = o.get_species(0)
    pmass = species_pmass(0)
    n, ek, ekmax, psig, nde = o.envar_species(0, pmass)
    rek, rmax, rps, rnde = numpy_envar_species(p, part, pmass)
    assert n == part.shape[0]
    assert np.allclose(ek, rek, rtol=1e-12, atol=1e-12 * np.abs(rek).max())
    assert ekmax == rmax > 0
    assert np.allclose(psig, rps, rtol=1e-12, atol=0)
    assert np.array_equal(nde, rnde) and nde.sum() > 0
    if ndim == 3:
        assert ek[3] != 0.0  # angular momentum of the laser-driven electrons
    energy, fmax, e2max = o.envar_fields()
    f = o.get_fields()
    sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2) if ndim == 3 else slice(0, 1))
    dg = p.dx * p.dy * (p.dz if ndim == 3 else p.dy)
    for c in range(p.nfield):
        fc = f[sl + (c,)]
        assert energy[c] == pytest.approx(dg * (fc * fc).sum(), rel=1e-12)
        assert fmax[c] == np.abs(fc).max()
    nc = 3 if ndim == 3 else 2
    assert e2max == pytest.approx((f[sl + (slice(0, nc),)] ** 2).sum(axis=-1).max(), rel=1e-15)


def test_host_envar_units():
    p, o = _state(3)
    pavg, favg, nde = envar(o, p, np_per_cell=4.0)
    n, ek, ekmax, psig, h = o.envar_species(0, ELECTRON_MASS)
    assert pavg[0, 0] == 4.0 * MEV_TO_JOULE * (ELECTRON_MASS * ek[6])
    assert pavg[1, 0] == ELECTRON_MASS * ekmax
    assert pavg[3, 0] == ELECTRON_MASS * (ek[0] * (1.0 / n))
    assert pavg[9, 0] == (1.0 / n) * ek[5] < 0  # electrons
    energy, fmax, _ = o.envar_fields()
    assert favg[0] == FIELD_ENERGY * energy[0] and favg[4] == ELECTRON_MASS * fmax[1]
    assert np.array_equal(nde[:, 0], h)
