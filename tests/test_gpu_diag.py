"""agpu_diag (Envar / energy_momenta, src/diagnostics/diag_part_and_fields.f90:
172-220, 485-719) against numpy sums over the state the device returns, for
both forms, after steps that gave the particles momenta (and, in the split
form, left removed records stored behind the alive ones).

* FP64 form: every sum within 1e-12 (relative).
* FP32 split form: the per-record terms are formed in FP32 (the records'
  own precision) and summed in FP64: kinetic energy, momenta and field
  energies within 1e-6, charge within 1e-12 (exact terms).
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.sim import PicDevice, unpack_slot
from tests.helpers import laser_fields, plasma_source, small_case

pytestmark = pytest.mark.gpu


def _run(ndim, precision, steps=8):
    p = small_case(ndim, precision=precision)
    dev = PicDevice(p)
    dev.set_fields(laser_fields(p, a0=4.0))
    dev.set_plasma_source(plasma_source(p))
    dev.load_plasma(0)
    t = 0.0
    for it in range(steps):
        dev.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    return p, dev


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("precision,tol", [(AGPU_FP64, 1e-12), (AGPU_FP32_SPLIT, 1e-6)])
@pytest.mark.parametrize("steps", [8, 11, 12])
def test_diag_sums(ndim, precision, tol, steps):
    """After 8 and 12 steps removed records of the last pushes are still
    stored behind the alive ones; after 11 the last step shifted the window
    (removal and injection after the push)."""
    p, dev = _run(ndim, precision, steps)
    d = dev.diag()
    s = dev.get_species(0)
    f = dev.get_fields()
    q, _, w = unpack_slot(s[:, -1])
    w = w.astype(np.float64)
    pm = s[:, ndim:2 * ndim] if ndim == 3 else np.column_stack([s[:, 2], s[:, 3], np.zeros(len(s))])
    gam = np.sqrt(1.0 + np.sum(pm * pm, axis=1))
    kin = np.sum(w * (gam - 1.0))
    assert kin > 0.0
    assert d.np[0] == len(s)
    assert abs(d.kin_energy[0] - kin) <= tol * kin
    assert abs(d.charge[0] - np.sum(q * w)) <= 1e-12 * abs(np.sum(q * w))
    scale = np.sum(w * np.sqrt(np.sum(pm * pm, axis=1)))
    for c in range(3):
        assert abs(d.momentum[0][c] - np.sum(w * pm[:, c])) <= tol * scale, c
    sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2) if ndim == 3 else slice(0, 1))
    dv = p.dx * p.dy * (p.dz if ndim == 3 else 1.0)
    for c in range(p.nfield):
        ref = np.sum(f[sl + (c,)] ** 2) * dv
        assert abs(d.field_energy[c] - ref) <= tol * max(ref, 1e-30), c
    ne = 3 if ndim == 3 else 2
    emax = max(np.abs(f[sl + (c,)]).max() for c in range(ne))
    assert abs(d.max_abs_e - emax) <= 1e-12 * emax


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("precision,tol", [(AGPU_FP64, 1e-12), (AGPU_FP32_SPLIT, 1e-6)])
def test_diag_sums_fresh_records(ndim, precision, tol):
    """Records set from the host (a count that is not a multiple of four,
    random momenta, no removed records): the straight pass over the arrays."""
    from aladyn_b200.sim import pack_slot
    p = small_case(ndim, precision=precision)
    dev = PicDevice(p)
    rng = np.random.default_rng(5)
    n = 40_003
    nd = 2 * ndim + 1
    rec = np.zeros((n, nd))
    lo = (p.xmn + 3 * p.dx, p.ymn + 3 * p.dy, p.zmn + 3 * p.dz)
    hi = (p.xmn + (p.nx - 3) * p.dx, p.ymn + (p.ny - 3) * p.dy, p.zmn + (p.nz - 3) * p.dz)
    for d in range(ndim):
        rec[:, d] = rng.uniform(lo[d], hi[d], n)
    rec[:, ndim:2 * ndim] = rng.normal(0.0, 0.5, (n, ndim))
    rec[:, -1] = pack_slot(rng.integers(-1, 3, n), 0, rng.uniform(0.1, 2.0, n))
    dev.set_species(0, rec)
    d = dev.diag()
    s = dev.get_species(0)
    q, _, w = unpack_slot(s[:, -1])
    w = w.astype(np.float64)
    pm = s[:, ndim:2 * ndim]
    kin = np.sum(w * (np.sqrt(1.0 + np.sum(pm * pm, axis=1)) - 1.0))
    assert d.np[0] == n
    assert abs(d.kin_energy[0] - kin) <= tol * kin
    assert abs(d.charge[0] - np.sum(q * w)) <= 1e-12 * np.sum(np.abs(q) * w)
    scale = np.sum(w * np.sqrt(np.sum(pm * pm, axis=1)))
    for c in range(ndim):
        assert abs(d.momentum[0][c] - np.sum(w * pm[:, c])) <= tol * scale, c
