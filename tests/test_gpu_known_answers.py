"""The schemes' known answers on the device, in both precision forms (the
CPU tests hold the oracle to the same answers):

* field solver: a vacuum pulse's energy centroid moves at the Yee scheme's
  group velocity from its numerical dispersion relation, der_ord 2 and 3,
  to 1 % of the 3-4 % slowdown (tests/test_oracle_dispersion.py);
* push: a particle at the relativistic E x B drift velocity moves
  uniformly; the rotation angle per step in a uniform B is the implicit
  equation's closed form; the uniform-E momentum ramp
  (tests/test_oracle_push.py);
* gather: fields linear in x, y, z are gathered exactly at each
  component's staggered nodes (tests/test_oracle_gather.py).

Tolerances: the FP64 form as the oracle's (1e-13 or tighter); the FP32
split form to its FP32 round-off (1e-5 relative, 1e-4 for B recovered from
the rotation, where p^{n+1/2} - p^{n-1/2} loses a decade); a half-cell
stagger error would show at about 3e-3."""
import math

import numpy as np
import pytest

from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
from aladyn_b200.config import Grid, make_params
from aladyn_b200.sim import PicDevice, pack_slot, unpack_slot
from tests.helpers import small_case
from tests.test_oracle_dispersion import CASES, _centroid, _ks, _predicted, _pulse
from tests.test_oracle_gather import STAGGER2, STAGGER3, _expected, _linear, _particles

pytestmark = pytest.mark.gpu

FORMS = [AGPU_FP64, AGPU_FP32_SPLIT]
REL = {AGPU_FP64: 1e-13, AGPU_FP32_SPLIT: 1e-5}


@pytest.mark.parametrize("precision", FORMS)
@pytest.mark.parametrize("ndim", [2, 3])
def test_device_group_velocity(ndim, precision):
    c = CASES[ndim]
    for der_ord in (2, 3):
        g = Grid(ndim, c["nx"], c["ntr"], c["ntr"], k0=10.0, yx_rat=4.0, zx_rat=4.0, cfl=0.8)
        p = make_params(g, precision=precision, w_sh=0, capacity=(16, 0, 0, 0), der_ord=der_ord)
        ebf, x = _pulse(p, p.xmn + 0.25 * c["nx"] * p.dx, c["length"], c["w0"])
        dev = PicDevice(p)
        dev.set_fields(ebf)
        c0 = _centroid(p, dev.get_fields(), x)
        t = 0.0
        for it in range(c["steps"]):
            out = dev.lp_run(t, it)
            assert out.error_bits == 0
            t += p.dt
        v = (_centroid(p, dev.get_fields(), x) - c0) / (c["steps"] * p.dt)
        dev.close()
        vp = _predicted(p, ebf[2:c["nx"] + 2, 2:c["ntr"] + 2, _ks(p), 1])
        print(f"{ndim}D der_ord {der_ord} precision {precision}: measured {v:.7f} predicted {vp:.7f}")
        assert abs(v - vp) <= 0.01 * (1.0 - vp), (der_ord, v, vp)


def _device(ndim, precision, fields, p_init):
    p = small_case(ndim, precision=precision, nx=64, ny=32, nz=32, cap=16, w_sh=0)
    dev = PicDevice(p)
    ebf = np.zeros(dev.field_shape(), order="F")
    for comp, val in fields.items():
        ebf[..., comp] = val
    dev.set_fields(ebf)
    rec = np.zeros((1, 2 * ndim + 1), order="F")
    rec[0, 0] = 0.4 * p.nx * p.dx
    rec[0, ndim:2 * ndim] = p_init[:ndim]
    rec[0, -1] = pack_slot(-1, 0, 0.0)  # an electron of zero weight
    dev.set_species(0, rec)
    return p, dev, rec


def _history(p, dev, rec, steps):
    hist = [rec[0].copy()]
    t = 0.0
    for it in range(1, steps + 1):
        out = dev.lp_run(t, it)
        assert out.error_bits == 0
        q = dev.get_species(0)
        assert q.shape[0] == 1
        hist.append(q[0].copy())
        t += p.dt
    dev.close()
    return np.array(hist)


def _comps(ndim):
    return (0, 1, 2) if ndim == 2 else (0, 1, 5)


@pytest.mark.parametrize("precision", FORMS)
@pytest.mark.parametrize("ndim", [2, 3])
def test_device_drift_rotation_and_ramp(ndim, precision):
    rel = REL[precision]
    ex, ey, bz = _comps(ndim)
    # relativistic E x B drift: no force at v = E0 / B0
    e0, b0 = 2.7, 3.0
    v = e0 / b0
    gam = 1.0 / math.sqrt(1.0 - v * v)
    p, dev, rec = _device(ndim, precision, {ey: e0, bz: b0}, [gam * v, 0.0, 0.0])
    h = _history(p, dev, rec, 12)
    assert np.abs(h[:, ndim] - gam * v).max() <= rel * gam * v
    assert np.abs(h[:, ndim + 1:2 * ndim]).max() <= rel * gam * v
    assert np.abs(np.diff(h[:, 0]) - p.dt * v).max() <= 10 * rel * p.dt
    # rotation in a uniform Bz
    b0 = 40.0
    p0 = np.array([0.6, -0.8, 0.0]) * 1.5
    p, dev, rec = _device(ndim, precision, {bz: b0}, p0)
    h = _history(p, dev, rec, 12)
    big_p = np.linalg.norm(p0)
    b = 0.5 * p.dt * b0
    c2 = (-(1 + b * b - big_p ** 2) + math.sqrt((1 + b * b - big_p ** 2) ** 2 + 4 * big_p ** 2)) / (2 * big_p ** 2)
    theta = 2.0 * math.acos(math.sqrt(c2))
    mom = h[:, ndim:ndim + 2]
    step = np.diff(np.unwrap(np.arctan2(mom[:, 1], mom[:, 0])))
    assert np.abs(step - theta).max() <= 10 * rel
    assert np.abs(np.linalg.norm(mom, axis=1) - big_p).max() <= 10 * rel * big_p
    # uniform-E ramp
    e0 = 3.0
    p, dev, rec = _device(ndim, precision, {ex: e0}, [0.1, 0.0, 0.0])
    h = _history(p, dev, rec, 15)
    px = 0.1 - np.arange(16) * p.dt * e0
    assert np.abs(h[:, ndim] - px).max() <= 10 * rel * np.abs(px).max()


def _by_index(rec):
    _, ind, _ = unpack_slot(rec[:, -1])
    return rec[np.argsort(ind)]


def _gather_case(ndim, precision, n, rng, mom, fields):
    p = small_case(ndim, precision=precision, nx=48, ny=32, nz=32, cap=4096, w_sh=0)
    rec = _particles(p, n, rng, mom)
    rec[:, -1] = pack_slot(-1, np.arange(n), 0.0)  # part_ind identifies the record
    dev = PicDevice(p)
    f = np.zeros(dev.field_shape(), order="F")
    for comp, coef in fields.items():
        stag = (STAGGER3 if ndim == 3 else STAGGER2)[comp]
        f[..., comp] = _linear(p, comp, stag, coef, f.shape)
    dev.set_fields(f)
    dev.set_species(0, rec)
    out = dev.lp_run(0.0, 1)
    assert out.error_bits == 0
    got = _by_index(dev.get_species(0))
    dev.close()
    assert got.shape == rec.shape
    return p, rec, got


@pytest.mark.parametrize("precision", FORMS)
@pytest.mark.parametrize("ndim", [2, 3])
def test_device_gathers_linear_fields_exactly(ndim, precision):
    rel = REL[precision]
    rng = np.random.default_rng(11)
    coefs = {c: rng.uniform(-0.4, 0.4, 4) for c in range(ndim)}
    p, rec, got = _gather_case(ndim, precision, 2000, rng, 0.0, coefs)
    for c in range(ndim):
        e = -got[:, ndim + c] / p.dt
        want = _expected(p, coefs[c], rec)
        assert np.abs(e - want).max() <= 10 * rel * np.abs(want).max(), c
    comps = [2] if ndim == 2 else [3, 4, 5]
    for comp in comps:
        axis = comp - 3 if ndim == 3 else 2
        mom = rng.normal(0.0, 0.8, (2000, 3))
        mom[:, axis] = 0.0
        coef = np.array([3.0, *rng.uniform(-0.6, 0.6, 3)])
        p, rec, got = _gather_case(ndim, precision, 2000, rng, mom[:, :ndim], {comp: coef})
        p0 = np.zeros((2000, 3))
        p1 = np.zeros((2000, 3))
        p0[:, :ndim] = rec[:, ndim:2 * ndim]
        p1[:, :ndim] = got[:, ndim:2 * ndim]
        d = p1 - p0
        s = (p1 + p0) / np.sqrt(1.0 + (0.25 * (p1 + p0) ** 2).sum(axis=1))[:, None]
        bvec = -np.cross(s, d) / (s ** 2).sum(axis=1)[:, None]
        bgot = bvec[:, axis] / (-0.5 * p.dt)
        want = _expected(p, coef, rec)
        tol = (1e-11 if precision == AGPU_FP64 else 1e-4) * np.abs(want).max()
        assert np.abs(bgot - want).max() <= tol, comp
