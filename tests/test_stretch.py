"""Stretched transverse grids (str_flag 1, 2: set_grid, src/grid/
set_grid_param.f90:52-226; the particle maps of src/grid/stretched_grid.f90;
the metric factors in rote/rotb, ef_bds/bf_bds and curr_mpi_collect) in the
host restatement and the oracle, on CPU.

* The grid: ny_stretch = nint(ny/6) (str_flag 1) or nint(ny/4) (2) cells at
  each end; the uniform middle keeps y(i) = dy (i - 1 - ny/2) and metric 1;
  the stretched cells grow monotonically towards the ends.
* The particle map sends every node y(i) to i - 1 (its cell coordinate on
  the uniform computational grid) in all three zones, to round-off.
* Fields in vacuum: a stretched run and a uniform run of the oracle agree
  bit for bit on the nodes that the stretched ends cannot have reached (the
  metric is exactly 1 there and the update is the same arithmetic).
"""
import numpy as np
import pytest

from aladyn_b200.config import StretchedGrid
from oracle.oracle import Oracle
from tests.helpers import laser_fields, small_case


@pytest.mark.parametrize("ndim,str_flag", [(2, 1), (2, 2), (3, 1)])
def test_grid_and_metric(ndim, str_flag):
    p = small_case(ndim, nx=32, ny=48, nz=24)
    ny = p.ny
    dy = p.dy
    sg = StretchedGrid(p, str_flag)
    ns = sg.n_stretch
    assert ns == int(np.floor(ny * (1 / 6 if str_flag == 1 else 0.25) + 0.5))
    y = sg.y["y"]
    # uniform middle, metric 1
    mid = np.arange(ns + 1, ny + 2 - ns)
    assert np.array_equal(y[mid], dy * (mid - 1 - ny // 2).astype(float))
    # (the half node above smax = y(ny + 1 - ns) is already stretched)
    assert (sg.y["d1"][mid] == 1.0).all() and (sg.y["d1h"][mid[:-1]] == 1.0).all()
    assert sg.y["d1h"][mid[-1]] < 1.0
    # stretched ends: strictly increasing, cells growing towards the ends
    assert (np.diff(y) > 0).all()
    cells = np.diff(y)
    assert (np.diff(cells[:ns + 1]) < 0).all() and (np.diff(cells[ny - ns:]) > 0).all()
    assert (sg.y["d1"] > 0).all() and (sg.y["d1"] <= 1.0).all()
    # the box bounds follow the stretched ends
    assert p.gymin == y[1] and p.gymax == y[ny + 1] and p.ymn == y[1]
    assert p.gymax - p.gymin > ny * dy


@pytest.mark.parametrize("ndim,str_flag", [(2, 1), (3, 2)])
def test_map_sends_nodes_to_cell_index(ndim, str_flag):
    p = small_case(ndim, nx=32, ny=48, nz=24)
    sg = StretchedGrid(p, str_flag)
    axes = [("y", sg.y, p.ny)] + ([("z", sg.z, p.nz)] if ndim == 3 else [])
    for name, ax, n in axes:
        for i in range(1, n + 2):
            assert abs(sg.map(name, ax["y"][i]) - (i - 1)) < 1e-9, (name, i)
        # half nodes map half way
        for i in range(1, n + 1):
            assert abs(sg.map(name, ax["yh"][i]) - (i - 0.5)) < 1e-9, (name, i)


@pytest.mark.parametrize("ndim", [2, 3])
def test_vacuum_fields_match_uniform_away_from_the_ends(ndim):
    steps = 6
    p0 = small_case(ndim, nx=48, ny=48, nz=48, w_sh=0)
    ps = small_case(ndim, nx=48, ny=48, nz=48, w_sh=0)
    sg = StretchedGrid(ps, 1)
    ebf = laser_fields(p0, a0=1.0, w0=0.12 * p0.ny * p0.dy)
    uni, st = Oracle(p0), Oracle(ps)
    st.set_stretch(sg)
    uni.set_fields(ebf)
    st.set_fields(ebf)
    t = 0.0
    for it in range(steps):
        assert uni.lp_run(t, it)[0] == 0 and st.lp_run(t, it)[0] == 0
        t += p0.dt
    fu, fs = uni.get_fields(), st.get_fields()
    ns = sg.n_stretch
    m = ns + steps + 4  # rows (and planes) the stretched ends can have reached, with margin
    sl = (slice(3, p0.nx), slice(2 + m, p0.ny + 2 - m),
          slice(2 + m, p0.nz + 2 - m) if ndim == 3 else slice(0, 1))
    assert np.abs(fu[sl]).max() > 0.1
    assert np.array_equal(fu[sl], fs[sl])
    # and they do differ near the stretched ends
    assert not np.array_equal(fu, fs)
