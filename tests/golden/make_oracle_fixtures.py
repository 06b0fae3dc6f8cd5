"""Regression fixtures of the oracle (not outputs of the reference, which
cannot be built here): small seeded runs whose results the oracle must keep
reproducing bit for bit, so that an edit of the oracle that changes its
arithmetic is caught.  Each case stores SHA-256 digests of the FP64 bit
patterns of its outputs and a few summary values for reading.

Regenerate (only after an intended change of the oracle's arithmetic):
    python tests/golden/make_oracle_fixtures.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return hashlib.sha256(a.view(np.uint64).tobytes()).hexdigest()


def lwfa_case(ndim, steps=6):
    from oracle.oracle import Oracle
    from tests.helpers import laser_fields, plasma_source, small_case
    p = small_case(ndim, nx=32, ny=16, nz=12, cap=60_000)
    o = Oracle(p)
    o.set_fields(laser_fields(p))
    o.set_plasma_source(plasma_source(p))
    o.load_plasma(0)
    t = 0.0
    for it in range(steps):
        rc, out = o.lp_run(t, it, initial_time=(it == 0))
        assert rc == 0
        t += p.dt
    f, s, j = o.get_fields(), o.get_species(0), o.get_currents()
    return {"fields": digest(f), "species": digest(s), "currents": digest(j), "np": int(s.shape[0]),
            "field_l2": [float(np.linalg.norm(f[..., c])) for c in range(f.shape[-1])]}


def ionization_case():
    from oracle.oracle import build_ionization_table
    tab, de_inv = build_ionization_table(7, 0, 1, 0.5, 0.03)
    return {"table": digest(tab), "de_inv": float(de_inv), "shape": list(tab.shape)}


def cases():
    return {"lwfa2d_32x16_6steps": lwfa_case(2), "lwfa3d_32x16x12_6steps": lwfa_case(3),
            "adk_nitrogen_model1": ionization_case()}


if __name__ == "__main__":
    with open(os.path.join(HERE, "oracle_fixtures.json"), "w") as f:
        json.dump(cases(), f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", os.path.join(HERE, "oracle_fixtures.json"))
