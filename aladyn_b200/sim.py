"""Python host side of the B200 PIC step: a thin object over the C-ABI.

``PicDevice`` owns one library handle.  Its methods are the calls the
reference's Fortran driver makes around the PIC step, with the reference's
names where one exists:

* ``lp_run(t, iter)``  – one call of ``lp_run`` (src/dynamics/
  pic_evolve_in_time.f90:113-144): ``lpf2_evolve`` plus the window shift;
* ``set_fields`` / ``get_fields`` – the module array ``ebf(n1p,n2p,n3p,nf)``;
* ``set_species`` / ``get_species`` – ``spec(ic)%part(np, ndv)``;
* ``diag()`` – the FP64 energy/charge reductions of ``Envar``.

Arrays are numpy arrays in the reference's Fortran (column-major) layout.
There is no CPU fallback: without the device library every call raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import AGPU_E_INDEX, AgpuDiagOut, AgpuStepOut, AgpuTimers, check
from .config import dims, ndv


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def pack_slot(charge, part_ind, wgh) -> np.ndarray:
    """Pack int16 charge | int16 part_ind | float32 wgh into FP64 slots
    (the ``equivalence`` of src/work/precision_def.F90:33-40)."""
    charge = np.asarray(charge, dtype=np.int16)
    part_ind = np.asarray(part_ind, dtype=np.int16)
    wgh = np.asarray(wgh, dtype=np.float32)
    charge, part_ind, wgh = np.broadcast_arrays(charge, part_ind, wgh)
    b = (charge.astype(np.uint16).astype(np.uint64)
         | (part_ind.astype(np.uint16).astype(np.uint64) << np.uint64(16))
         | (wgh.view(np.uint32).astype(np.uint64) << np.uint64(32)))
    return b.view(np.float64)


def unpack_slot(slot: np.ndarray):
    b = np.ascontiguousarray(slot, dtype=np.float64).view(np.uint64)
    charge = (b & np.uint64(0xFFFF)).astype(np.uint16).view(np.int16)
    part_ind = ((b >> np.uint64(16)) & np.uint64(0xFFFF)).astype(np.uint16).view(np.int16)
    wgh = (b >> np.uint64(32)).astype(np.uint32).view(np.float32)
    return charge, part_ind, wgh


class PicDevice:
    """One simulation resident on one GPU."""

    def __init__(self, params, lib_path: str | None = None, handle=None):
        self.lib = abi.load_library(lib_path)
        self.params = params
        self.owned = handle is None
        if handle is None:
            self.h = C.c_void_p()
            check(self.lib.agpu_create(C.byref(params), C.byref(self.h)), "agpu_create")
        else:
            self.h = handle  # an instance of a PicBatch, destroyed with the batch
        self.n1p, self.n2p, self.n3p = dims(params)
        self.ndv = ndv(params)
        self.nf = params.nfield
        self.nc = params.curr_ndim

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if self.h and self.owned:
            self.lib.agpu_destroy(self.h)
        self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- fields ------------------------------------------------------------
    def field_shape(self):
        return (self.n1p, self.n2p, self.n3p, self.nf)

    def set_fields(self, ebf: np.ndarray):
        a = np.asfortranarray(ebf, dtype=np.float64)
        assert a.shape == self.field_shape(), a.shape
        check(self.lib.agpu_set_fields(self.h, _dptr(a), self.n1p, self.n2p, self.n3p, self.nf),
              "agpu_set_fields")

    def get_fields(self) -> np.ndarray:
        a = np.zeros(self.field_shape(), dtype=np.float64, order="F")
        check(self.lib.agpu_get_fields(self.h, _dptr(a), self.n1p, self.n2p, self.n3p, self.nf),
              "agpu_get_fields")
        return a

    def get_currents(self) -> np.ndarray:
        a = np.zeros((self.n1p, self.n2p, self.n3p, self.nc), dtype=np.float64, order="F")
        check(self.lib.agpu_get_currents(self.h, _dptr(a), self.n1p, self.n2p, self.n3p, self.nc),
              "agpu_get_currents")
        return a

    # -- particles ---------------------------------------------------------
    def set_species(self, ic: int, part: np.ndarray):
        a = np.asfortranarray(part, dtype=np.float64)
        assert a.ndim == 2 and a.shape[1] == self.ndv, a.shape
        check(self.lib.agpu_set_species(self.h, ic, _dptr(a), a.shape[0], a.shape[0], self.ndv),
              "agpu_set_species")

    def count(self, ic: int) -> int:
        n = C.c_int64()
        check(self.lib.agpu_get_count(self.h, ic, C.byref(n)), "agpu_get_count")
        return n.value

    def get_species(self, ic: int) -> np.ndarray:
        n = self.count(ic)
        a = np.zeros((max(n, 1), self.ndv), dtype=np.float64, order="F")
        got = C.c_int64()
        check(self.lib.agpu_get_species(self.h, ic, _dptr(a), a.shape[0], C.byref(got), self.ndv),
              "agpu_get_species")
        return a[:n]

    def window_inject(self, ic: int, part: np.ndarray):
        a = np.asfortranarray(part, dtype=np.float64)
        check(self.lib.agpu_window_inject(self.h, ic, _dptr(a), a.shape[0], a.shape[0], self.ndv),
              "agpu_window_inject")

    # -- PWFA bunch set-up (beam_inject) ---------------------------------------
    def beam_inject(self, ic: int, part: np.ndarray, gam0: float) -> int:
        """Append the bunch records inside the box to species ic and add the
        bunch fields (Poisson solve of the bunch charge).  Returns the status:
        0, or AGPU_E_INDEX when a record's stencil left the array."""
        a = np.asfortranarray(part, dtype=np.float64)
        rc = self.lib.agpu_beam_inject(self.h, ic, _dptr(a), a.shape[0], a.shape[0], self.ndv, gam0)
        if rc not in (0, AGPU_E_INDEX):
            check(rc, "agpu_beam_inject")
        return rc

    def beam_potential(self, rho: np.ndarray, gam2: float) -> np.ndarray:
        """fft_3d_psolv / fft_2d_psolv of rho(n1p, n2p, n3p) on the device."""
        a = np.asfortranarray(rho, dtype=np.float64)
        assert a.shape == (self.n1p, self.n2p, self.n3p)
        out = np.zeros_like(a, order="F")
        check(self.lib.agpu_beam_potential(self.h, _dptr(a), _dptr(out), gam2), "agpu_beam_potential")
        return out

    # -- initial state on the device ----------------------------------------
    def set_plasma_source(self, src):
        check(self.lib.agpu_set_plasma_source(self.h, C.byref(src)), "agpu_set_plasma_source")

    def load_plasma(self, ic: int):
        check(self.lib.agpu_load_plasma(self.h, ic), "agpu_load_plasma")

    def init_laser(self, laser):
        check(self.lib.agpu_init_laser(self.h, C.byref(laser)), "agpu_init_laser")

    def init_lp_fields(self, pulse):
        check(self.lib.agpu_init_lp_fields(self.h, C.byref(pulse)), "agpu_init_lp_fields")

    def set_ionization_species(self, ic, atomic_number, ion_min, ion_max, model, lp_max):
        check(self.lib.agpu_set_ionization_species(self.h, ic, atomic_number, ion_min, ion_max,
                                                   model, lp_max), "agpu_set_ionization_species")

    def set_ionization_table(self, ic, table: np.ndarray, de_inv: float):
        a = np.asfortranarray(table, dtype=np.float64)
        check(self.lib.agpu_set_ionization_table(self.h, ic, _dptr(a), a.shape[0] - 2, a.shape[1] - 1,
                                                 de_inv), "agpu_set_ionization_table")

    # -- the step ------------------------------------------------------------
    def lp_run(self, t: float, iteration: int, initial_time: bool = False) -> AgpuStepOut:
        out = AgpuStepOut()
        check(self.lib.agpu_step(self.h, iteration, t, 1 if initial_time else 0, C.byref(out)),
              "agpu_step")
        return out

    step = lp_run

    # -- envelope cycle (Env_cycle, src/ALaDyn.F90:111-130) -------------------
    def set_stretch(self, st):
        """A stretched grid (config.stretched_grid); st keeps its metric
        arrays alive until the call returns (the library copies them)."""
        check(self.lib.agpu_set_stretch(self.h, C.byref(st.struct)), "agpu_set_stretch")

    def env_enable(self, ep: "abi.AgpuEnvParams"):
        check(self.lib.agpu_env_enable(self.h, C.byref(ep)), "agpu_env_enable")

    def init_envelope(self, pulse, plane_wave: bool = False):
        check(self.lib.agpu_init_envelope(self.h, C.byref(pulse), 1 if plane_wave else 0), "agpu_init_envelope")

    def set_envelope(self, env: np.ndarray):
        a = np.asfortranarray(env, dtype=np.float64)
        assert a.shape == (self.n1p, self.n2p, self.n3p, 4), a.shape
        check(self.lib.agpu_set_envelope(self.h, _dptr(a), self.n1p, self.n2p, self.n3p, 4), "agpu_set_envelope")

    def get_envelope(self) -> np.ndarray:
        a = np.zeros((self.n1p, self.n2p, self.n3p, 4), dtype=np.float64, order="F")
        check(self.lib.agpu_get_envelope(self.h, _dptr(a), self.n1p, self.n2p, self.n3p, 4), "agpu_get_envelope")
        return a

    def get_env_source(self) -> np.ndarray:
        nav = 4 if self.n3p > 1 else 3
        a = np.zeros((self.n1p, self.n2p, self.n3p, nav), dtype=np.float64, order="F")
        check(self.lib.agpu_get_env_source(self.h, _dptr(a), self.n1p, self.n2p, self.n3p, nav),
              "agpu_get_env_source")
        return a

    def env_run(self, t: float, iteration: int) -> AgpuStepOut:
        out = AgpuStepOut()
        check(self.lib.agpu_env_run(self.h, iteration, t, C.byref(out)), "agpu_env_run")
        return out

    def diag(self) -> AgpuDiagOut:
        out = AgpuDiagOut()
        check(self.lib.agpu_diag(self.h, C.byref(out)), "agpu_diag")
        return out

    # -- control / profiling --------------------------------------------------
    def envar_species(self, ic: int, pmass: float) -> "abi.AgpuEnvarOut":
        o = abi.AgpuEnvarOut()
        check(self.lib.agpu_envar_species(self.h, ic, pmass, C.byref(o)), "agpu_envar_species")
        return o

    def envar_fields(self) -> "abi.AgpuEnvarFieldsOut":
        o = abi.AgpuEnvarFieldsOut()
        check(self.lib.agpu_envar_fields(self.h, C.byref(o)), "agpu_envar_fields")
        return o

    def set_deterministic(self, on: bool = True):
        check(self.lib.agpu_set_deterministic(self.h, 1 if on else 0), "agpu_set_deterministic")

    def set_profiling(self, on: bool = True):
        check(self.lib.agpu_set_profiling(self.h, 1 if on else 0), "agpu_set_profiling")

    def timers(self) -> AgpuTimers:
        t = AgpuTimers()
        check(self.lib.agpu_get_timers(self.h, C.byref(t)), "agpu_get_timers")
        return t

    def reset_timers(self):
        check(self.lib.agpu_reset_timers(self.h), "agpu_reset_timers")

    def stream(self) -> int:
        s = C.c_void_p()
        check(self.lib.agpu_get_stream(self.h, C.byref(s)), "agpu_get_stream")
        return s.value or 0

    def synchronize(self):
        check(self.lib.agpu_synchronize(self.h), "agpu_synchronize")


    def set_deferred_counts(self, on: bool = True):
        check(self.lib.agpu_set_deferred_counts(self.h, 1 if on else 0), "agpu_set_deferred_counts")

    def set_fused_yee(self, on: bool = True):
        check(self.lib.agpu_set_fused_yee(self.h, 1 if on else 0), "agpu_set_fused_yee")

    def window_state(self):
        """(xlapse, nptx[4], sptx_max[4], xmn): what a dump carries besides
        fields and particles."""
        x = C.c_double()
        n = (C.c_int64 * 4)()
        m = (C.c_int64 * 4)()
        xmn = C.c_double()
        check(self.lib.agpu_get_window_state(self.h, C.byref(x), n, m, C.byref(xmn)), "agpu_get_window_state")
        return x.value, list(n), list(m), xmn.value

    def set_window_state(self, xlapse: float, nptx):
        n = (C.c_int64 * 4)(*[int(v) for v in (list(nptx) + [0, 0, 0, 0])[:4]])
        check(self.lib.agpu_set_window_state(self.h, float(xlapse), n), "agpu_set_window_state")

    def set_sort_interval(self, steps: int):
        """Move the records along the tile permutation every `steps` steps (0: never)."""
        check(self.lib.agpu_set_sort_interval(self.h, int(steps)), "agpu_set_sort_interval")

    def set_step_graphs(self, on: bool = True):
        check(self.lib.agpu_set_step_graphs(self.h, 1 if on else 0), "agpu_set_step_graphs")


class PicBatch:
    """N independent simulations on one GPU (a parameter scan), advanced
    together by agpu_batch_run.  ``instances[i]`` is a PicDevice view of
    instance i for its set-up and read-back."""

    def __init__(self, params_list, lib_path: str | None = None):
        self.lib = abi.load_library(lib_path)
        n = len(params_list)
        self._params = (abi.AgpuParams * n)(*params_list)
        self.b = C.c_void_p()
        check(self.lib.agpu_batch_create(C.cast(self._params, C.c_void_p), n, C.byref(self.b)), "agpu_batch_create")
        self.instances = []
        for i in range(n):
            h = C.c_void_p()
            check(self.lib.agpu_batch_handle(self.b, i, C.byref(h)), "agpu_batch_handle")
            self.instances.append(PicDevice(self._params[i], lib_path, handle=h))

    def __len__(self):
        return len(self.instances)

    def run(self, nsteps: int, nthreads: int = 0):
        """Advance every instance by nsteps; returns the per-instance status."""
        st = (C.c_int32 * len(self))()
        self.lib.agpu_batch_run(self.b, nsteps, nthreads, st)
        return list(st)

    def set_graphs(self, on: bool = True):
        check(self.lib.agpu_batch_set_graphs(self.b, 1 if on else 0), "agpu_batch_set_graphs")

    def set_multi(self, on: bool = True):
        check(self.lib.agpu_batch_set_multi(self.b, 1 if on else 0), "agpu_batch_set_multi")

    def launches(self) -> int:
        n = C.c_int64()
        check(self.lib.agpu_batch_launches(self.b, C.byref(n)), "agpu_batch_launches")
        return n.value

    def clock(self, i: int):
        it, t = C.c_int32(), C.c_double()
        check(self.lib.agpu_batch_clock(self.b, i, C.byref(it), C.byref(t)), "agpu_batch_clock")
        return it.value, t.value

    def close(self):
        if self.b:
            for d in self.instances:
                d.h = C.c_void_p()
            self.lib.agpu_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_lp_cycle(dev: PicDevice, nsteps: int, t0: float = 0.0, iter0: int = 0):
    """Mirror of Lp_cycle (src/ALaDyn.F90:89-107) for nsteps iterations:
    lp_run, then t += dt and iter += 1; the first call is the initial time."""
    dt = dev.params.dt
    t, it = t0, iter0
    outs = []
    for _ in range(nsteps):
        outs.append(dev.lp_run(t, it, initial_time=(t < dt)))
        t = t + dt
        it = it + 1
    return outs, t, it
