"""Envar (src/diagnostics/diag_part_and_fields.f90:485-719) on the host from
the device's reductions (agpu_envar_species, agpu_envar_fields): the same
quantities, in the same units, that the reference stores in pavg(1:11,
nst, ic), favg(1:12, nst) and nde(1:ne, nst, ic) for one diagnostic call,
single domain (the allreduces are identities).

pavg(:, ic): 1 total energy (J) = np_per_cell * mev_to_joule * pmass *
sum wgh (gamma-1); 2 max energy (MeV) = pmass * max(gamma-1); 3 total
angular momentum = mev_to_joule * pmass * sum wgh (y pz - z py) (3D); 4-6
averaged momenta (MeV/c) = pmass * ek(k)/np (3D unweighted, 2D weighted
sums, as energy_momenta forms them); 7-9 1e3 * pmass * sum (p_k -
<p_k>)^2 / np; 10 mean charge = sum charge wgh / np; 11 charge per cell
= sum charge wgh / (nx ny nz).  favg: 1-3 E energies and 7-9 B energies (J)
= field_energy * dgvol * sum F^2; 4-6 and 10-12 e0 * max |F| (TV/m).
"""
from __future__ import annotations

import numpy as np

from .config import PROTON_MASS_NORM

ELECTRON_MASS = 0.510998928   # MeV, src/work/phys_param.f90:47
MEV_TO_JOULE = 1.602e-13      # diag_part_and_fields.f90:492
FIELD_ENERGY = 1.156e-06      # diag_part_and_fields.f90:493
NE = 100


def species_pmass(ic: int, mass_number=(1.0, 1.0, 1.0)) -> float:
    """pmass = electron_mass * mass(ic) (MeV), mass(1) = 1 (electrons),
    mass(ic) = mass_number(ic-1) * proton_mass_norm (set_init_param.f90:198-201)."""
    return ELECTRON_MASS * (1.0 if ic == 0 else mass_number[ic - 1] * PROTON_MASS_NORM)


def envar(holder, p, mass_number=(1.0, 1.0, 1.0), np_per_cell: float = 1.0):
    """pavg (11, nsp), favg (12,), nde (NE, nsp) of one Envar call on a state
    holder with envar_species(ic, pmass) / envar_fields() (the device's
    PicDevice or the oracle)."""
    nsp = int(p.nsp)
    ndim = int(p.ndim)
    cnd = 3 if ndim == 3 else 2
    ncells = float(p.nx * p.ny * (p.nz if ndim == 3 else 1))
    pavg = np.zeros((11, nsp))
    nde = np.zeros((NE, nsp))
    for ic in range(nsp):
        pmass = species_pmass(ic, mass_number)
        np_, ek, ekmax, psig, h = _species(holder, ic, pmass)
        np_norm = 1.0 / np_ if np_ > 0 else 1.0
        ek_max = pmass * ekmax
        pavg[0, ic] = np_per_cell * MEV_TO_JOULE * (pmass * ek[6])
        pavg[1, ic] = ek_max
        pavg[2, ic] = MEV_TO_JOULE * (pmass * ek[3])
        pavg[3:6, ic] = pmass * np.array([ek[k] * np_norm if k < cnd else 0.0 for k in range(3)])
        pavg[6:6 + cnd, ic] = 1.e+03 * pmass * (np_norm * psig[:cnd])
        pavg[9, ic] = np_norm * ek[5]
        pavg[10, ic] = (1. / ncells) * ek[5]
        nde[:, ic] = h
    energy, fmax, _ = _fields(holder)
    favg = np.zeros(12)
    favg[0:3] = FIELD_ENERGY * energy[0:3]
    favg[6:9] = FIELD_ENERGY * energy[3:6]
    favg[3:6] = ELECTRON_MASS * fmax[0:3]
    favg[9:12] = ELECTRON_MASS * fmax[3:6]
    return pavg, favg, nde


def _species(holder, ic, pmass):
    r = holder.envar_species(ic, pmass)
    if isinstance(r, tuple):
        return r
    return int(r.np), np.array(r.ek[:]), float(r.ekmax), np.array(r.psig[:]), np.array(r.nde[:])


def _fields(holder):
    r = holder.envar_fields()
    if isinstance(r, tuple):
        return r
    return np.array(r.energy[:]), np.array(r.fmax[:]), float(r.e2max)
