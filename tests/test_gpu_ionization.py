"""Field ionization on the device against the oracle: a laser crosses a
nitrogen dopant (neutral atoms, 7 levels, one-level ADK model 1, N2 -> two
electrons' weight per ion) plus a pre-ionised electron background.

* FP64 form, deterministic mode: new-electron counts per step, every ion's
  charge state and every electron record bit-exact after 12 steps (same
  Philox draws, same FP64 table).
* FP32 split form: total new electrons within 3% of the FP64 oracle (the
  ionization index nint(de_inv*|E|) moves across table bins when |E| is
  gathered in FP32).
"""
import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.sim import PicDevice, unpack_slot
from oracle.oracle import Oracle
from tests.helpers import LAM0, laser_fields, plasma_source, small_case

pytestmark = pytest.mark.gpu

A0 = 1.0
LP_MAX = 1.5 * A0 * 2 * np.pi / LAM0


def _case(precision):
    kw = dict(nx=48, ny=24, nz=16, cap=400_000, nsp=2, ionz_lev=1, n_mol_atoms=(1, 2, 1, 1))
    p = small_case(3, precision=precision, **kw)
    dev = PicDevice(p)
    ora = Oracle(small_case(3, precision=AGPU_FP64, **kw))
    ebf = laser_fields(p, a0=A0)
    el = plasma_source(p, ic=0, npx=1, npy=1, npz=1, n_over_n0=8.71, x_start_frac=0.3)
    ion = plasma_source(p, ic=1, npx=1, npy=1, npz=1, charge=0, wgh=0.0435, x_start_frac=0.3, seed=4242)
    for s in (dev, ora):
        s.set_fields(ebf)
        s.set_plasma_source(el)
        s.set_plasma_source(ion)
        s.load_plasma(0)
        s.load_plasma(1)
    dev.set_ionization_species(1, 7, 0, 7, 1, LP_MAX)
    ora.set_ionization_species(1, 7, 0, 1, LP_MAX)
    return p, dev, ora


def test_fp64_ionization_bitexact():
    p, dev, ora = _case(AGPU_FP64)
    dev.set_deterministic(True)
    t, total = 0.0, 0
    for it in range(12):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        assert out.new_electrons == oo.new_electrons, (it, out.new_electrons, oo.new_electrons)
        assert out.np[0] == oo.np[0] and out.np[1] == oo.np[1]
        total += out.new_electrons
        t += p.dt
    assert total > 1000  # the laser did ionize
    for ic in (0, 1):
        a, b = dev.get_species(ic), ora.get_species(ic)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), ic
    q, _, _ = unpack_slot(dev.get_species(1)[:, -1])
    assert q.max() >= 2  # several levels crossed


def test_fp32_split_ionization_statistics():
    p, dev, ora = _case(AGPU_FP32_SPLIT)
    t, n32, n64 = 0.0, 0, 0
    for it in range(12):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert out.error_bits == 0
        n32 += out.new_electrons
        n64 += oo.new_electrons
        t += p.dt
    assert n64 > 1000
    assert abs(n32 - n64) <= 0.03 * n64, (n32, n64)
    q32, _, _ = unpack_slot(dev.get_species(1)[:, -1])
    q64, _, _ = unpack_slot(ora.get_species(1)[:, -1])
    assert abs(int(q32.astype(np.int64).sum()) - int(q64.astype(np.int64).sum())) <= 0.03 * int(q64.sum())


@pytest.mark.parametrize("dopant", [0.005, 0.01])
def test_fp32_split_ionization_binomial_bound(dopant):
    """The split form against the FP64 oracle on a larger box at the C4
    workload's dopant fractions (0.5% and 1% of the electron density), with a
    bound tied to the count: each ion's ionization is a Bernoulli draw, so a
    total of n new electrons has a variance of at most n; the two runs draw
    independently (their records are ordered differently), so
    |n32 - n64| <= 5 sqrt(2 n64) unless the FP32 gather biases the rates."""
    kw = dict(nx=96, ny=32, nz=24, cap=1_200_000, nsp=2, ionz_lev=1, n_mol_atoms=(1, 2, 1, 1))
    p = small_case(3, precision=AGPU_FP32_SPLIT, **kw)
    dev = PicDevice(p)
    ora = Oracle(small_case(3, precision=AGPU_FP64, **kw), threads=8)
    ebf = laser_fields(p, a0=A0)
    n_e = 8.71
    el = plasma_source(p, ic=0, npx=1, npy=1, npz=1, n_over_n0=n_e, x_start_frac=0.3)
    ion = plasma_source(p, ic=1, npx=2, npy=1, npz=1, charge=0, wgh=dopant * n_e / 2, x_start_frac=0.3, seed=4242)
    for s in (dev, ora):
        s.set_fields(ebf)
        s.set_plasma_source(el)
        s.set_plasma_source(ion)
        s.load_plasma(0)
        s.load_plasma(1)
    dev.set_ionization_species(1, 7, 0, 7, 1, LP_MAX)
    ora.set_ionization_species(1, 7, 0, 1, LP_MAX)
    t, n32, n64 = 0.0, 0, 0
    for it in range(12):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        rc, oo = ora.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0 and out.error_bits == 0
        n32 += out.new_electrons
        n64 += oo.new_electrons
        t += p.dt
    print(f"dopant {dopant}: new electrons FP32 {n32}, FP64 {n64}, bound {5 * np.sqrt(2 * n64):.0f}")
    assert n64 > 5000
    assert abs(n32 - n64) <= 5 * np.sqrt(2 * n64), (n32, n64)
