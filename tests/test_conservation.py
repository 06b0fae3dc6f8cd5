"""Discrete continuity of a whole step on the oracle, through the host-side
residual of aladyn_b200.conservation (the same check the GPU tests and the
benchmark apply to the device's currents): after a few laser-driven steps,
one more step's currents satisfy rho1 - rho0 + c div J_raw = 0 to FP64
round-off, c = 1/2 (2D) or 1/3 (3D) (grid_part_connect.f90:956-1334 with
the djc normalisation of set_init_param.f90:92-103)."""
import numpy as np
import pytest

from aladyn_b200.conservation import charge_density, step_residual
from oracle.oracle import Oracle
from tests.helpers import laser_fields, plasma_source, small_case


def conservation_case(ndim, precision=0, nx=48, ny=24, nz=24):
    """A laser in a plasma slab kept 6 cells away from every edge (no
    removal, no folded ghost current), no moving window."""
    p = small_case(ndim, precision=precision, nx=nx, ny=ny, nz=nz, cap=200_000, w_sh=0)
    src = plasma_source(p, x_start_frac=0.15)
    src.x_end = p.xmax - 6 * p.dx
    src.y_min, src.y_max = p.gymin + 6 * p.dy, p.gymax - 6 * p.dy
    if ndim == 3:
        src.z_min, src.z_max = p.gzmin + 6 * p.dz, p.gzmax - 6 * p.dz
    return p, src, laser_fields(p, a0=3.0)


def residual_after(holder, p, steps):
    t = 0.0
    for it in range(steps):
        holder.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    part0 = holder.get_species(0)
    holder.lp_run(t, steps)
    part1 = holder.get_species(0)
    assert part1.shape[0] == part0.shape[0] > 0
    return step_residual(p, part0, part1, holder.get_currents(), margin=4)


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_step_conserves_charge(ndim):
    p, src, ebf = conservation_case(ndim)
    o = Oracle(p)
    o.set_fields(ebf)
    o.set_plasma_source(src)
    o.load_plasma(0)
    res, rho, divj = residual_after(o, p, 4)
    assert divj > 1e-4 * rho  # the step moved charge
    assert res <= 1e-14 * rho, (res, rho, divj)


def test_charge_density_partition_of_unity():
    p, src, _ = conservation_case(3)
    o = Oracle(p)
    o.set_plasma_source(src)
    o.load_plasma(0)
    part = o.get_species(0)
    rho = charge_density(p, part, (o.n1p, o.n2p, o.n3p))
    from aladyn_b200.sim import unpack_slot
    q, _, w = unpack_slot(part[:, -1])
    total = float(np.sum(q.astype(np.float32) * w.astype(np.float32), dtype=np.float64))
    assert abs(rho.sum() - total) <= 1e-12 * abs(total)


@pytest.mark.parametrize("shape", [0, 1])
@pytest.mark.parametrize("edge", [6.0, 0.6])
@pytest.mark.parametrize("ndim", [2, 3])
def test_total_current_is_the_charge_weighted_displacement(ndim, edge, shape):
    """The first moment of the qden shapes is the particle's position, so
    the Esirkepov current of a step, summed over the grid, is exactly
    sum_p w_p (x1_p - x0_p) per axis, w = real(charge * wgh, sp): the raw
    sum of a component is (ndim) w dx_inv displacement (the transverse
    shape factors of each term sum to ndim), and djc = dx / ndim scales it
    back (grid_part_connect.f90:979-1059, 1168-1334; set_init_param.f90:
    92-103).  With the plasma 0.6 cells from the transverse edges the
    particles deposit into the ghost layers, and the sum holds through the
    fold of those layers into the boundary cells (jc_xyzbd,
    mpi_curr_interface.f90:551-643).  The cubic extension's 4-point shapes
    (shape 1) have the same first moment and obey the same identity."""
    from aladyn_b200.sim import unpack_slot
    p, src, ebf = conservation_case(ndim)
    p.shape = shape
    src.y_min, src.y_max = p.gymin + edge * p.dy, p.gymax - edge * p.dy
    if ndim == 3:
        src.z_min, src.z_max = p.gzmin + edge * p.dz, p.gzmax - edge * p.dz
    o = Oracle(p)
    o.set_fields(ebf)
    o.set_plasma_source(src)
    o.load_plasma(0)
    t = 0.0
    for it in range(4):
        o.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
    part0 = o.get_species(0)
    o.lp_run(t, 4)
    part1 = o.get_species(0)
    assert part1.shape[0] == part0.shape[0] > 0
    q, _, wgh = unpack_slot(part1[:, -1])
    w = (q.astype(np.float32) * wgh.astype(np.float32)).astype(np.float64)
    jc = o.get_currents()
    for a in range(ndim):
        moved = w * (part1[:, a] - part0[:, a])
        total = float(np.sum(jc[..., a]))
        scale = float(np.sum(np.abs(moved)))
        assert scale > 0
        assert abs(total - float(np.sum(moved))) <= 1e-13 * scale, (a, total, np.sum(moved), scale)
