"""PWFA electron bunch records, as the reference's start-up builds them.

``bunch_parameters`` restates the bunch block of ``set_initial_param``
(src/start/set_init_param.f90:342-370): gam0, bet0, the Gaussian bunch
volume, the density ratio rhob, the macro-particles per cell and the
macro-particle weight jb_norm.  ``bunch_records`` restates ``beam_data``
(src/IO/init_beam_part_distrib.f90:43-110) with ``bunch_gen``
(src/work/util.f90:274-414): Gaussian x, y, z, py, pz, a uniform px spread of
rms 0.01 dg gam around gam, re-centring on the sample means, shifts to the
bunch centre, and the packed slot (charge = electron_charge_norm = -1,
part_ind = bunch index, wgh = real(jb_norm, sp)).

The reference draws from gfortran's ``random_number`` seeded from
/dev/urandom (not reproducible); here the draws are Philox4x32-10 (counter =
(n, n >> 32, block, 0x42554e43), key = seed) with Box-Muller Gaussians, the
same distributions.  The records are host data: the host passes them to
``agpu_beam_inject`` (and the same array to any checker), as the reference's
pe0 builds the bunch on the host and distributes it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .lattice import philox4x32_10
from .sim import pack_slot

PI2 = 6.283185307179586          # src/work/phys_param.f90:28
E_CHARGE = 1.6021766 * 1.e-7     # e charge in pC, phys_param.f90:45
_TAG = 0x42554E43                # Philox counter word of the bunch draws


@dataclass
class Bunch:
    nb_tot: int            # macro-particles
    charge_pc: float       # bunch_charge (pC)
    sxb: float             # rms length along x (um)
    syb: float             # rms transverse size (um)
    gam: float             # gamma
    epsy: float            # transverse emittances (mm mrad = um)
    epsz: float
    dg: float              # energy spread (%)
    xc: float              # centre
    yc: float = 0.0
    zc: float = 0.0
    seed: int = 77


def bunch_parameters(p, b: Bunch, n0_ref: float) -> dict:
    """set_init_param.f90:350-370 for one bunch (ndim from the params)."""
    gam0 = b.gam
    u0_b = math.sqrt(gam0 * gam0 - 1.)
    bet0 = u0_b / gam0
    if p.ndim < 3:
        bunch_volume = PI2 * b.sxb * b.syb * p.dy
        gvol_inv = p.dx_inv * p.dy_inv * p.dy_inv
    else:
        bunch_volume = PI2 * math.sqrt(PI2) * b.sxb * b.syb * b.syb
        gvol_inv = p.dx_inv * p.dy_inv * p.dz_inv
    rhob = b.charge_pc / (E_CHARGE * bunch_volume)
    rhob = 1.e-06 * rhob / n0_ref
    ncell = bunch_volume * gvol_inv
    x = b.nb_tot / ncell
    nb_per_cell = int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)
    jb_norm = rhob / nb_per_cell if nb_per_cell > 0 else 1.
    return dict(gam0=gam0, bet0=bet0, bunch_volume=bunch_volume, rhob=rhob, nb_per_cell=nb_per_cell,
                jb_norm=jb_norm)


def _uniform(n: int, block: int, seed: int):
    """Four arrays of uniforms in (0, 1) from Philox block `block` of particles 0..n-1."""
    idx = np.arange(0, n, dtype=np.uint64)
    r = philox4x32_10((idx & np.uint64(0xFFFFFFFF)).astype(np.uint32), (idx >> np.uint64(32)).astype(np.uint32),
                      np.full(n, block, dtype=np.uint32), np.full(n, _TAG, dtype=np.uint32), seed, seed >> 32)
    return [(x.astype(np.float64) + 0.5) * (1.0 / 4294967296.0) for x in r]


def _gauss_pair(u1, u2):
    rr = np.sqrt(-2.0 * np.log(u1))
    return rr * np.cos(PI2 * u2), rr * np.sin(PI2 * u2)


def bunch_records(p, b: Bunch, n0_ref: float, part_ind: int = 1) -> np.ndarray:
    """Fortran-layout records part(nb_tot, ndv) of one bunch (beam_data + bunch_gen)."""
    ndim = p.ndim
    n = int(b.nb_tot)
    prm = bunch_parameters(p, b, n0_ref)
    gm = b.gam
    ua = _uniform(n, 0, b.seed)
    ub = _uniform(n, 1, b.seed)
    g_a, g_b = _gauss_pair(ua[0], ua[1])
    g_c, g_d = _gauss_pair(ua[2], ua[3])
    g_x, _ = _gauss_pair(ub[0], ub[1])
    a_px = 2.0 * ub[2] - 1.0                   # cut = 3: uniform on (-1, 1)
    nch = 2 * ndim + 1
    rec = np.zeros((n, nch), dtype=np.float64, order="F")
    if ndim == 2:
        sigs = (b.sxb, b.syb, math.sqrt(3.0) * 0.01 * b.dg * gm, b.epsy / b.syb)
        cols = (g_x, g_a, a_px, g_b)           # x, y, px, py
        for j in range(4):
            rec[:, j] = sigs[j] * cols[j]
        rec[:, 2] += gm
        mean = rec[:, :4].sum(axis=0) / float(n)
        rec[:, 0] -= mean[0]
        rec[:, 1] -= mean[1]
        rec[:, 2] -= (mean[2] - gm)
        rec[:, 3] -= mean[3]
        rec[:, 0] += b.xc
        rec[:, 1] += b.yc
    else:
        sigs = (b.sxb, b.syb, b.syb, math.sqrt(3.0) * 0.01 * b.dg * gm, b.epsy / b.syb, b.epsz / b.syb)
        cols = (g_x, g_a, g_c, a_px, g_b, g_d)  # x, y, z, px, py, pz
        for j in range(6):
            rec[:, j] = sigs[j] * cols[j]
        rec[:, 3] += gm
        mean = (1. / float(n)) * rec[:, :6].sum(axis=0)
        for j in range(6):
            rec[:, j] -= (mean[j] - gm) if j == 3 else mean[j]
        rec[:, 0] += b.xc
        rec[:, 1] += b.yc
        rec[:, 2] += b.zc
    wgh = np.float32(prm["jb_norm"])
    rec[:, nch - 1] = pack_slot(np.full(n, -1, dtype=np.int16), np.full(n, part_ind, dtype=np.int16),
                                np.full(n, wgh, dtype=np.float32))
    return rec


__all__ = ["Bunch", "bunch_parameters", "bunch_records"]
