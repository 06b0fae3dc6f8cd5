"""A known answer for the oracle's ionization cycle (set_ion_efield,
src/particles/grid_part_connect.f90:288-410; ionization_cycle and
part_ionize, src/ionization/ionize.f90:390-558; the electron injection
258-322): in a uniform field E0 every ion sees |E| = E0 exactly (the
gather's weights sum to one), so with one level per step (ionz_lev = 1) its
charge is a Markov chain that climbs from z to z + 1 with the table's
probability w(nk, z), nk = nint(de_inv E0).  After K steps the number of
ions at each charge is binomial with the chain's probabilities; the counts
of a seeded run fall within 5 sigma of them, the new electrons of each step
equal the charge the ions gained, and each carries the ion's weight times
n_mol_atoms.  Ions and electrons have zero weight, so no current disturbs
the field, and the ions sit 6 cells inside the box, beyond the reach of
the open boundaries' disturbance over the K steps."""
import math

import numpy as np

from aladyn_b200.sim import unpack_slot
from oracle.oracle import Oracle
from tests.helpers import plasma_source, small_case

K = 3


def test_charge_states_follow_the_table_chain():
    p = small_case(3, nx=48, ny=24, nz=16, cap=400_000, nsp=2, ionz_lev=1, n_mol_atoms=(1, 2, 1, 1), w_sh=0)
    o = Oracle(p)
    lp_max = 12.0
    e0 = 0.0125 * lp_max  # the first two levels in play: w(0) = 0.94, w(1) = 0.027
    ebf = np.zeros(o.field_shape(), order="F")
    ebf[..., 0] = e0
    o.set_fields(ebf)
    ion = plasma_source(p, ic=1, npx=2, npy=2, npz=2, charge=0, wgh=0.0, x_start_frac=0.2, seed=4242)
    ion.x_end = p.xmax - 6 * p.dx
    ion.y_min, ion.y_max = p.gymin + 6 * p.dy, p.gymax - 6 * p.dy
    ion.z_min, ion.z_max = p.gzmin + 6 * p.dz, p.gzmax - 6 * p.dz
    o.set_plasma_source(ion)
    o.load_plasma(1)
    o.set_ionization_species(1, 7, 0, 1, lp_max)
    n = o.count(1)
    assert n > 5000
    tab = o.ionization_table(1, 7)
    de_inv = (tab.shape[0] - 2) / lp_max  # n_ge bins over (0, lp_max]
    nk = int(math.floor(de_inv * e0 + 0.5))
    w = tab[nk, :]
    assert 0.05 < w[0] < 0.95  # the first level is neither sure nor impossible
    # the chain's distribution after each step
    dist = np.zeros(8)
    dist[0] = 1.0
    t = 0.0
    gained_before = 0
    for it in range(K):
        rc, out = o.lp_run(t, it + 1)
        assert rc == 0
        t += p.dt
        nxt = dist * (1 - w)
        nxt[1:] += (dist * w)[:-1]
        dist = nxt
        q, _, _ = unpack_slot(o.get_species(1)[:, -1])
        counts = np.bincount(q.astype(np.int64), minlength=8)
        for z in range(4):
            mean = n * dist[z]
            sigma = math.sqrt(max(n * dist[z] * (1 - dist[z]), 1.0))
            assert abs(counts[z] - mean) <= 5 * sigma, (it, z, counts[z], mean, sigma)
        gained = int(q.astype(np.int64).sum())
        assert out.new_electrons == gained - gained_before
        gained_before = gained
    el = o.get_species(0)
    assert el.shape[0] == gained_before > 0
    qe, _, we = unpack_slot(el[:, -1])
    assert (qe == -1).all() and (we == 0.0).all()
    assert np.abs(el[:, 3:6]).max() < 1.0  # born at rest, then accelerated by E0 only
