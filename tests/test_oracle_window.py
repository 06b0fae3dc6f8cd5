"""A known answer for the oracle's moving window with injection
(lp_window_xshift, particles_inject, add_particles: src/dynamics/
window.f90:39-347; cell_part_dist, src/parallel/mpi_part_interface.f90:
549-597): a jitter-free lattice plasma at rest in zero fields stays at rest,
and after the window has moved by more than the plasma's initial offset
every cell column of the window holds the lattice's own number of
particles, the columns injected at each shift included: no gap and no
overlap at the seams between loaded and injected columns, whatever the
shift sizes (nint rounding gives 7 or 8 cells here)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.helpers import plasma_source, small_case


@pytest.mark.parametrize("ndim", [2, 3])
def test_injected_columns_continue_the_lattice(ndim):
    p = small_case(ndim, nx=64, ny=32, nz=16, w_sh=10)
    src = plasma_source(p, x_start_frac=0.25, jitter=0.0)
    o = Oracle(p)
    o.set_fields(np.zeros(o.field_shape(), order="F"))
    o.set_plasma_source(src)
    o.load_plasma(0)
    part0 = o.get_species(0)
    cells0 = np.floor((part0[:, 0] - o.xmn()) / p.dx).astype(np.int64)
    per_column = np.bincount(cells0)[cells0.max() - 1]  # a full column of the loaded lattice
    assert per_column > 0
    t, shifts = 0.0, []
    for it in range(60):
        rc, out = o.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0
        shifts.append(out.nshx)
        t += p.dt
    moved = sum(shifts)
    assert moved > 0.25 * p.nx and sorted(set(s for s in shifts if s)) == [7, 8]
    part = o.get_species(0)
    assert np.abs(part[:, ndim:2 * ndim]).max() == 0.0
    cells = np.floor((part[:, 0] - o.xmn()) / p.dx).astype(np.int64)
    hist = np.bincount(cells, minlength=p.nx)
    last = int(np.floor((p.xmax - p.xmn) / p.dx)) - 1  # the last full cell below xmax
    assert (hist[:last + 1] == per_column).all(), hist
    assert part.shape[0] == per_column * (last + 1)
