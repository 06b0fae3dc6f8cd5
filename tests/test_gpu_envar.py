"""The device's Envar reductions (agpu_envar_species / agpu_envar_fields)
against the oracle's restatement of Envar, energy_momenta and energy_spect
(src/diagnostics/diag_part_and_fields.f90:126-142, 172-220, 485-719):

* FP64 form in deterministic mode (particles and fields bit-exact with the
  oracle after the steps): sums within 1e-12 (the device sums with
  atomics, in another order), max(gamma - 1), the field maxima and all 100
  spectrum bins exact;
* FP32 split form: against the same formulas in numpy on the device's own
  records (agpu_get_species), sums within 1e-12, maxima and bins exact;
* the host's Envar in the reference's units from either holder agrees.
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.diagnostics import envar, species_pmass
from aladyn_b200.sim import PicDevice
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case
from tests.test_envar import numpy_envar_species

pytestmark = pytest.mark.gpu


def _pair(ndim, precision, steps=6):
    kw = dict(nx=48, ny=24, nz=16, cap=200_000, w_sh=0)
    p = small_case(ndim, precision=precision, **kw)
    dev = PicDevice(p)
    ora = Oracle(small_case(ndim, **kw))
    ebf = laser_fields(p, a0=3.0)
    src = plasma_source(p, x_start_frac=0.3)
    for s in (dev, ora):
        s.set_fields(ebf)
        s.set_plasma_source(src)
        s.load_plasma(0)
    if precision == AGPU_FP64:
        dev.set_deterministic(True)
    t = 0.0
    for it in range(steps):
        dev.lp_run(t, it, initial_time=(it == 0))
        ora.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    return p, dev, ora


@pytest.mark.parametrize("ndim", [2, 3])
def test_envar_fp64_matches_oracle(ndim):
    p, dev, ora = _pair(ndim, AGPU_FP64)
    assert np.array_equal(dev.get_species(0).view(np.uint64), ora.get_species(0).view(np.uint64))
    pmass = species_pmass(0)
    d = dev.envar_species(0, pmass)
    n, ek, ekmax, psig, nde = ora.envar_species(0, pmass)
    assert d.np == n > 0
    assert np.allclose(np.array(d.ek[:]), ek, rtol=1e-12, atol=1e-12 * np.abs(ek).max())
    assert d.ekmax == ekmax
    assert np.allclose(np.array(d.psig[:]), psig, rtol=1e-12, atol=0)
    assert np.array_equal(np.array(d.nde[:]), nde) and nde.sum() > 0
    fe = dev.envar_fields()
    energy, fmax, e2max = ora.envar_fields()
    assert np.allclose(np.array(fe.energy[:]), energy, rtol=1e-12, atol=0)
    assert np.array_equal(np.array(fe.fmax[:]), fmax) and fe.e2max == e2max
    pa, fa, na = envar(dev, p, np_per_cell=4.0)
    pb, fb, nb = envar(ora, p, np_per_cell=4.0)
    assert np.allclose(pa, pb, rtol=1e-12, atol=1e-12 * np.abs(pb).max())
    assert np.allclose(fa, fb, rtol=1e-12, atol=0) and np.array_equal(na, nb)
    dev.close()


@pytest.mark.parametrize("ndim", [2, 3])
def test_envar_split_form_matches_records(ndim):
    p, dev, _ = _pair(ndim, AGPU_FP32_SPLIT)
    part = dev.get_species(0)
    pmass = species_pmass(0)
    d = dev.envar_species(0, pmass)
    ek, ekmax, psig, nde = numpy_envar_species(p, part, pmass)
    assert d.np == part.shape[0]
    assert np.allclose(np.array(d.ek[:]), ek, rtol=1e-12, atol=1e-12 * np.abs(ek).max())
    assert d.ekmax == ekmax
    assert np.allclose(np.array(d.psig[:]), psig, rtol=1e-12, atol=0)
    assert np.array_equal(np.array(d.nde[:]), nde)
    dev.close()
