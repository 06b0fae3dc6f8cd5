"""ctypes wrapper of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg, never by the product package.  See aladyn_oracle.c for the
restated reference functions; parity unpinned (the Fortran reference cannot
be compiled here and ships no golden vectors).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    src = [os.path.join(HERE, f) for f in ("aladyn_oracle.c", "philox.h", "Makefile")]
    if force or not os.path.exists(LIB) or max(os.path.getmtime(s) for s in src) > os.path.getmtime(LIB):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "liboracle.so"], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = C.CDLL(LIB)
    P, D, I64 = C.c_void_p, C.POINTER(C.c_double), C.c_int64
    sig = {
        "ora_create": (P, [P]),
        "ora_destroy": (None, [P]),
        "ora_set_threads": (None, [P, C.c_int]),
        "ora_dims": (C.c_int, [P, C.POINTER(C.c_int)]),
        "ora_set_fields": (C.c_int, [P, D]),
        "ora_get_fields": (C.c_int, [P, D]),
        "ora_get_currents": (C.c_int, [P, D]),
        "ora_set_currents": (None, [P, D]),
        "ora_set_species": (C.c_int, [P, C.c_int, D, I64, I64]),
        "ora_get_species": (C.c_int, [P, C.c_int, D, I64, C.POINTER(I64)]),
        "ora_count": (I64, [P, C.c_int]),
        "ora_error_bits": (C.c_uint32, [P]),
        "ora_xmn": (C.c_double, [P]),
        "ora_get_window_state": (None, [P, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "ora_set_window_state": (None, [P, C.c_double, C.POINTER(C.c_int64)]),
        "ora_step": (C.c_int, [P, C.c_int, C.c_double, C.c_int, P]),
        "ora_field_bd": (None, [P]),
        "ora_advance_fields": (None, [P]),
        "ora_field_xadvect_once": (None, [P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
        "ora_curr_fold": (None, [P]),
        "ora_zero_currents": (None, [P]),
        "ora_deposit_move": (None, [P, D, D, C.c_float]),
        "ora_rho_one": (None, [P, D, D, C.c_double]),
        "ora_phase_gather_push": (None, [P, C.c_int, C.c_int]),
        "ora_get_scratch": (C.c_int, [P, C.c_int, D, I64]),
        "ora_shape_qlh": (None, [C.c_double, D, D, C.POINTER(C.c_int)]),
        "ora_shape_qqh": (None, [C.c_double, D, D, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "ora_shape_qden": (None, [C.c_double, D, C.POINTER(C.c_int)]),
        "ora_shape_cubic": (None, [C.c_double, D, D, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "ora_set_plasma_source": (C.c_int, [P, P]),
        "ora_load_plasma": (C.c_int, [P, C.c_int]),
        "ora_build_ionization_table": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, D, D]),
        "ora_set_ionization_species": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]),
        "ora_get_ionization_table": (C.c_int, [P, C.c_int, D]),
        "ora_ionz_de_inv": (C.c_double, [P, C.c_int]),
        "ora_draw": (C.c_double, [C.c_uint64, I64, C.c_int, C.c_int]),
        "ora_philox": (None, [C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]),
        "ora_beam_inject": (C.c_int, [P, C.c_int, D, I64, I64, C.c_double]),
        "ora_beam_potential": (C.c_int, [P, D, C.c_double]),
        "ora_grid_charge": (None, [P, D, I64, I64, D]),
        "ora_init_lp_fields": (None, [P, P]),
        "ora_envar_species": (None, [P, C.c_int, C.c_double, D]),
        "ora_envar_fields": (None, [P, D]),
        "ora_env_enable": (C.c_int, [P, P]),
        "ora_set_envelope": (C.c_int, [P, D]),
        "ora_get_envelope": (C.c_int, [P, D]),
        "ora_get_env_source": (C.c_int, [P, D]),
        "ora_init_envelope": (None, [P, P, C.c_int]),
        "ora_env_run": (C.c_int, [P, C.c_int, C.c_double, P]),
        "ora_set_stretch": (C.c_int, [P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


NGE = 10000


class Oracle:
    """The oracle's simulation state, same calls as aladyn_b200.sim.PicDevice."""

    def __init__(self, params, threads: int = 1):
        self.lib = load()
        self.params = params
        self._p = params  # keep alive
        self.h = self.lib.ora_create(C.byref(params))
        d = (C.c_int * 10)()
        self.lib.ora_dims(self.h, d)
        self.n1p, self.n2p, self.n3p = d[0], d[1], d[2]
        self.ix1, self.ix2, self.jy1, self.jy2, self.kz1, self.kz2 = d[3], d[4], d[5], d[6], d[7], d[8]
        self.ndv = d[9]
        self.nf = params.nfield
        self.nc = params.curr_ndim
        if threads > 1:
            self.lib.ora_set_threads(self.h, threads)

    def close(self):
        if self.h:
            self.lib.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field_shape(self):
        return (self.n1p, self.n2p, self.n3p, self.nf)

    def set_fields(self, ebf):
        a = np.asfortranarray(ebf, dtype=np.float64)
        assert a.shape == self.field_shape()
        self.lib.ora_set_fields(self.h, _dp(a))

    def set_stretch(self, st):
        """A stretched grid (aladyn_b200.config.stretched_grid)."""
        rc = self.lib.ora_set_stretch(self.h, C.cast(C.byref(st.struct), C.c_void_p))
        assert rc == 0, rc

    def field_xadvect(self, dth, v_adv, ic1, ic2, isch):
        """One field_xadvect pass (the comoving frame's x advection) on
        components ic1..ic2 (1-based); isch 0 explicit, 2 implicit."""
        self.lib.ora_field_xadvect_once(self.h, dth, v_adv, ic1, ic2, isch)

    def envar_species(self, ic, pmass):
        """Envar's per-species reductions: (np, ek(1:7), ekmax, psig(1:3), nde(1:100))."""
        out = np.zeros(116)
        self.lib.ora_envar_species(self.h, ic, pmass, _dp(out))
        return self.count(ic), out[:7].copy(), float(out[7]), out[8:11].copy(), out[16:116].copy()

    def envar_fields(self):
        """Envar's field reductions: (energy[6], fmax[6], e2max)."""
        out = np.zeros(16)
        self.lib.ora_envar_fields(self.h, _dp(out))
        return out[:6].copy(), out[6:12].copy(), float(out[12])

    def init_lp_fields(self, pulse):
        """init_lp_inc0_fields: pulse is an aladyn_b200.abi.AgpuLpPulse."""
        self.lib.ora_init_lp_fields(self.h, C.cast(C.pointer(pulse), C.c_void_p))

    # ---- envelope cycle ------------------------------------------------
    def env_enable(self, ep):
        """Allocate env(n1p,n2p,n3p,4); ep is an aladyn_b200.abi.AgpuEnvParams."""
        assert self.lib.ora_env_enable(self.h, C.cast(C.pointer(ep), C.c_void_p)) == 0

    def init_envelope(self, pulse, plane_wave=False):
        """init_(gprof_)envelope_field: adds the pulse's A^n, A^{n-1} to env."""
        self.lib.ora_init_envelope(self.h, C.cast(C.pointer(pulse), C.c_void_p), 1 if plane_wave else 0)

    def set_envelope(self, env):
        a = np.asfortranarray(env, dtype=np.float64)
        assert a.shape == (self.n1p, self.n2p, self.n3p, 4)
        assert self.lib.ora_set_envelope(self.h, _dp(a)) == 0

    def get_envelope(self):
        a = np.zeros((self.n1p, self.n2p, self.n3p, 4), dtype=np.float64, order="F")
        assert self.lib.ora_get_envelope(self.h, _dp(a)) == 0
        return a

    def get_env_source(self):
        nav = 4 if self.n3p > 1 else 3
        a = np.zeros((self.n1p, self.n2p, self.n3p, nav), dtype=np.float64, order="F")
        assert self.lib.ora_get_env_source(self.h, _dp(a)) == 0
        return a

    def env_run(self, t, iteration):
        from aladyn_b200.abi import AgpuStepOut
        out = AgpuStepOut()
        rc = self.lib.ora_env_run(self.h, iteration, t, C.byref(out))
        return rc, out

    def get_fields(self):
        a = np.zeros(self.field_shape(), dtype=np.float64, order="F")
        self.lib.ora_get_fields(self.h, _dp(a))
        return a

    def get_currents(self):
        a = np.zeros((self.n1p, self.n2p, self.n3p, self.nc), dtype=np.float64, order="F")
        self.lib.ora_get_currents(self.h, _dp(a))
        return a

    def set_currents(self, jc):
        a = np.asfortranarray(jc, dtype=np.float64)
        self.lib.ora_set_currents(self.h, _dp(a))

    def set_species(self, ic, part):
        a = np.asfortranarray(part, dtype=np.float64)
        rc = self.lib.ora_set_species(self.h, ic, _dp(a), a.shape[0], a.shape[0])
        assert rc == 0, rc

    def count(self, ic):
        return self.lib.ora_count(self.h, ic)

    def get_species(self, ic):
        n = self.count(ic)
        a = np.zeros((max(n, 1), self.ndv), dtype=np.float64, order="F")
        got = C.c_int64()
        self.lib.ora_get_species(self.h, ic, _dp(a), a.shape[0], C.byref(got))
        return a[:n]

    def set_plasma_source(self, src):
        assert self.lib.ora_set_plasma_source(self.h, C.byref(src)) == 0

    def load_plasma(self, ic):
        assert self.lib.ora_load_plasma(self.h, ic) == 0

    def set_ionization_species(self, ic, an, ion_min, model, lp_max):
        assert self.lib.ora_set_ionization_species(self.h, ic, an, ion_min, model, lp_max) == 0

    def ionization_table(self, ic, zmax):
        t = np.zeros((NGE + 2, zmax + 1), dtype=np.float64, order="F")
        assert self.lib.ora_get_ionization_table(self.h, ic, _dp(t)) == 0
        return t

    def lp_run(self, t, iteration, initial_time=False):
        from aladyn_b200.abi import AgpuStepOut
        out = AgpuStepOut()
        rc = self.lib.ora_step(self.h, iteration, t, 1 if initial_time else 0, C.byref(out))
        return rc, out

    def beam_inject(self, ic, part, gam0):
        """beam_inject: append the bunch records inside the box, add the bunch
        fields to ebf; jc(1) holds the potential afterwards."""
        a = np.asfortranarray(part, dtype=np.float64)
        return self.lib.ora_beam_inject(self.h, ic, _dp(a), a.shape[0], a.shape[0], gam0)

    def beam_potential(self, rho, gam2):
        """fft_3d_psolv / fft_2d_psolv on rho(n1p,n2p,n3p); returns a copy with
        the interior replaced by the potential."""
        a = np.array(rho, dtype=np.float64, order="F", copy=True)
        assert a.shape == (self.n1p, self.n2p, self.n3p)
        assert self.lib.ora_beam_potential(self.h, _dp(a), gam2) == 0
        return a

    def grid_charge(self, part):
        """set_grid_charge of the records part(np, ndv) on a zero grid."""
        a = np.asfortranarray(part, dtype=np.float64)
        den = np.zeros((self.n1p, self.n2p, self.n3p), dtype=np.float64, order="F")
        self.lib.ora_grid_charge(self.h, _dp(a), a.shape[0], a.shape[0], _dp(den))
        return den

    def error_bits(self):
        return self.lib.ora_error_bits(self.h)

    def xmn(self):
        return self.lib.ora_xmn(self.h)

    def window_state(self):
        """(xlapse, nptx[4], sptx_max[4], xmn) of the window and the
        injection, as aladyn_b200.sim.PicDevice.window_state."""
        x = C.c_double()
        n = (C.c_int64 * 4)()
        m = (C.c_int64 * 4)()
        self.lib.ora_get_window_state(self.h, C.byref(x), n, m)
        return x.value, list(n), list(m), self.xmn()

    def set_window_state(self, xlapse, nptx):
        n = (C.c_int64 * 4)(*[int(v) for v in (list(nptx) + [0, 0, 0, 0])[:4]])
        self.lib.ora_set_window_state(self.h, float(xlapse), n)


def build_ionization_table(an, z0, model, e_max, dt):
    lib = load()
    t = np.zeros((NGE + 2, an + 1), dtype=np.float64, order="F")
    de = C.c_double()
    rc = lib.ora_build_ionization_table(an, z0, model, e_max, dt, _dp(t), C.byref(de))
    assert rc == 0, rc
    return t, de.value
