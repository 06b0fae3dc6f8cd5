"""iform = 2, the reference's non-conserving deposit (ncdef_2d_curr /
ncdef_3d_curr, src/particles/grid_part_connect.f90:1338-1512), in the
oracle: every particle deposits half of q w dt v on the qlh shapes at its old
and at its new position, and the shapes sum to one, so the currents of a
step summed over the grid equal sum_p q w (dt / gamma) p to round-off
(curr_mpi_collect leaves them unscaled when iform = 2, and the ghost fold
keeps the sums); with iform = 0 the same particles give the Esirkepov
currents instead."""
import numpy as np
import pytest

from aladyn_b200.config import make_params
from aladyn_b200.sim import pack_slot, unpack_slot
from oracle.oracle import Oracle
from tests.helpers import grid_small


def _case(ndim, iform, n=300, seed=3):
    g = grid_small(ndim, 48, 24, 16)
    p = make_params(g, capacity=(4000, 0, 0, 0), w_sh=0, iform=iform)
    o = Oracle(p)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 7 if ndim == 3 else 5), order="F")
    lo = [p.xmn + 6 * p.dx, p.ymn + 5 * p.dy, p.zmn + 5 * p.dz]
    hi = [p.xmn + (p.nx - 6) * p.dx, p.ymn + (p.ny - 5) * p.dy, p.zmn + (p.nz - 5) * p.dz]
    for d in range(ndim):
        rec[:, d] = rng.uniform(lo[d], hi[d], n)
        rec[:, ndim + d] = rng.normal(0.0, 0.5, n)
    rec[:, -1] = pack_slot(-1, 0, 0.37)
    o.set_species(0, rec)
    return p, o


@pytest.mark.parametrize("ndim", [2, 3])
def test_ncdef_total_current(ndim):
    p, o = _case(ndim, 2)
    rc, _ = o.lp_run(0.0, 1)
    assert rc == 0
    part = o.get_species(0)
    jc = o.get_currents()
    ch, _, w = unpack_slot(part[:, -1])
    wght = (ch.astype(np.float32) * w.astype(np.float32)).astype(np.float64)
    pv = part[:, ndim:2 * ndim]
    gam = np.sqrt(1.0 + (pv * pv).sum(axis=1))
    for c in range(ndim):
        want = (wght * (p.dt / gam) * pv[:, c]).sum()
        got = jc[..., c].sum()
        assert abs(got - want) <= 1e-12 * np.abs(wght * (p.dt / gam) * pv[:, c]).sum(), (c, got, want)


@pytest.mark.parametrize("ndim", [2, 3])
def test_ncdef_differs_from_esirkepov(ndim):
    """Same particles, same step: iform = 2 and iform = 0 move the particles
    identically but deposit different currents."""
    p2, o2 = _case(ndim, 2)
    p0, o0 = _case(ndim, 0)
    assert o2.lp_run(0.0, 1)[0] == 0 and o0.lp_run(0.0, 1)[0] == 0
    assert np.array_equal(o2.get_species(0), o0.get_species(0))
    j2, j0 = o2.get_currents(), o0.get_currents()
    assert np.abs(j2 - j0).max() > 1e-3 * np.abs(j0).max()
