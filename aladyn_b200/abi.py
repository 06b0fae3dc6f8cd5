"""ctypes mirror of include/aladyn_gpu.h and the loader of the device library.

The structures below must match the C header byte for byte; the
``test_abi`` CPU test checks their sizes against the compiled library.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaladyn_gpu.so")

AGPU_OK = 0
AGPU_E_WINDOW = 2
AGPU_E_COUNT = 99
AGPU_E_ARG = 101
AGPU_E_CUDA = 102
AGPU_E_NOMEM = 103
AGPU_E_CAPACITY = 104
AGPU_E_INDEX = 105
AGPU_E_IONZ_INDEX = 106
AGPU_E_NONFINITE = 107
AGPU_E_NODEVICE = 108
AGPU_E_STATE = 109

AGPU_FP64 = 0
AGPU_FP32_SPLIT = 1

AGPU_SHAPE_QUADRATIC = 0
AGPU_SHAPE_CUBIC = 1

AGPU_EBIT_INDEX = 1
AGPU_EBIT_IONZ_INDEX = 2
AGPU_EBIT_NONFINITE = 4
AGPU_EBIT_CAPACITY = 8

# exchange points of a y slab's step (agpu_set_subdomain)
AGPU_HALO_FIELDS = 1
AGPU_HALO_PARTICLES = 2
AGPU_HALO_CURRENTS = 3
AGPU_HALO_E = 4
AGPU_HALO_B = 5
# int hook(void* user, agpu_handle* h, int32_t point, int32_t ic)
HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32)


class AgpuParams(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("nfield", C.c_int32),
        ("curr_ndim", C.c_int32),
        ("ibx", C.c_int32), ("iby", C.c_int32), ("ibz", C.c_int32),
        ("iform", C.c_int32),
        ("precision", C.c_int32),
        ("nsp", C.c_int32),
        ("nsp_run", C.c_int32),
        ("w_sh", C.c_int32),
        ("ionz_lev", C.c_int32),
        ("n_mol_atoms", C.c_int32 * 4),
        ("shape", C.c_int32),
        ("reserved_i", C.c_int32 * 3),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dx_inv", C.c_double), ("dy_inv", C.c_double), ("dz_inv", C.c_double),
        ("dt", C.c_double),
        ("xmn", C.c_double), ("ymn", C.c_double), ("zmn", C.c_double),
        ("gxmin", C.c_double), ("gxmax", C.c_double),
        ("gymin", C.c_double), ("gymax", C.c_double),
        ("gzmin", C.c_double), ("gzmax", C.c_double),
        ("xmax", C.c_double),
        ("se_coeff", C.c_double * 2),
        ("djc", C.c_double * 3),
        ("ompe", C.c_double),
        ("lorentz_fact", C.c_double * 4),
        ("w_speed", C.c_double), ("wi_time", C.c_double), ("wf_time", C.c_double),
        ("reserved_d", C.c_double * 4),
        ("seed", C.c_uint64),
        ("capacity", C.c_int64 * 4),
    ]


class AgpuPlasma(C.Structure):
    _fields_ = [
        ("ic", C.c_int32),
        ("npx", C.c_int32), ("npy", C.c_int32), ("npz", C.c_int32),
        ("charge", C.c_int32),
        ("part_ind", C.c_int32),
        ("wgh", C.c_float),
        ("reserved_f", C.c_float),
        ("x_start", C.c_double), ("x_end", C.c_double),
        ("y_min", C.c_double), ("y_max", C.c_double),
        ("z_min", C.c_double), ("z_max", C.c_double),
        ("jitter", C.c_double),
        ("seed", C.c_uint64),
    ]


class AgpuLaser(C.Structure):
    _fields_ = [
        ("a0", C.c_double), ("lam0", C.c_double), ("w0_y", C.c_double),
        ("tau_fwhm", C.c_double), ("xc", C.c_double), ("xf", C.c_double),
        ("y0", C.c_double), ("z0", C.c_double),
    ]


class AgpuLpPulse(C.Structure):
    _fields_ = [
        ("ee0", C.c_double), ("t_loc", C.c_double), ("tf", C.c_double), ("wx", C.c_double),
        ("wy", C.c_double), ("xf0", C.c_double), ("om0", C.c_double), ("ycent", C.c_double),
        ("zcent", C.c_double), ("g_prof", C.c_int32), ("reserved", C.c_int32),
    ]


class AgpuEnvParams(C.Structure):
    _fields_ = [
        ("om0", C.c_double), ("opt_der1", C.c_double), ("hord_der2", C.c_double),
        ("der_ord", C.c_int32), ("reserved", C.c_int32),
    ]


class AgpuStretchAxis(C.Structure):
    _fields_ = [
        ("cnst", C.c_double), ("smin", C.c_double), ("smax", C.c_double), ("xs", C.c_double),
        ("dl_inv", C.c_double), ("dli_inv", C.c_double), ("ratio", C.c_double), ("nl_stretch", C.c_double),
        ("init_cell", C.c_double), ("n", C.c_int32), ("reserved", C.c_int32),
        ("d1", C.POINTER(C.c_double)), ("d1h", C.POINTER(C.c_double)),
    ]


class AgpuStretch(C.Structure):
    _fields_ = [("on", C.c_int32), ("reserved", C.c_int32), ("y", AgpuStretchAxis), ("z", AgpuStretchAxis)]


AGPU_NE = 100


class AgpuEnvarOut(C.Structure):
    _fields_ = [
        ("np", C.c_int64), ("ek", C.c_double * 7), ("ekmax", C.c_double), ("psig", C.c_double * 3),
        ("nde", C.c_double * AGPU_NE),
    ]


class AgpuEnvarFieldsOut(C.Structure):
    _fields_ = [("energy", C.c_double * 6), ("fmax", C.c_double * 6), ("e2max", C.c_double)]


class AgpuStepOut(C.Structure):
    _fields_ = [
        ("np", C.c_int64 * 4),
        ("removed", C.c_int64 * 4),
        ("injected", C.c_int64 * 4),
        ("new_electrons", C.c_int64),
        ("ion_field_max", C.c_double),
        ("xmn", C.c_double),
        ("nshx", C.c_int32),
        ("error_bits", C.c_uint32),
    ]


class AgpuDiagOut(C.Structure):
    _fields_ = [
        ("field_energy", C.c_double * 6),
        ("max_abs_e", C.c_double),
        ("kin_energy", C.c_double * 4),
        ("charge", C.c_double * 4),
        ("momentum", (C.c_double * 3) * 4),
        ("np", C.c_int64 * 4),
    ]


class AgpuTimers(C.Structure):
    _fields_ = [
        ("ms_push_deposit", C.c_double),
        ("ms_yee", C.c_double),
        ("ms_sort", C.c_double),
        ("ms_window", C.c_double),
        ("ms_ionize", C.c_double),
        ("ms_other", C.c_double),
        ("launches_push_deposit", C.c_int64),
        ("launches_yee", C.c_int64),
        ("launches_total", C.c_int64),
        ("pushes", C.c_int64),
        ("yee_cells", C.c_int64),
    ]


# Every exported symbol of the C-ABI, with its ctypes signature.
_P = C.c_void_p
_D = C.POINTER(C.c_double)
SIGNATURES = {
    "agpu_create": (C.c_int, [C.POINTER(AgpuParams), C.POINTER(_P)]),
    "agpu_destroy": (C.c_int, [_P]),
    "agpu_error_string": (C.c_char_p, [C.c_int]),
    "agpu_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "agpu_set_fields": (C.c_int, [_P, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "agpu_get_fields": (C.c_int, [_P, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "agpu_get_currents": (C.c_int, [_P, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "agpu_set_species": (C.c_int, [_P, C.c_int32, _D, C.c_int64, C.c_int64, C.c_int32]),
    "agpu_get_species": (C.c_int, [_P, C.c_int32, _D, C.c_int64, C.POINTER(C.c_int64), C.c_int32]),
    "agpu_get_count": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int64)]),
    "agpu_set_plasma_source": (C.c_int, [_P, C.POINTER(AgpuPlasma)]),
    "agpu_load_plasma": (C.c_int, [_P, C.c_int32]),
    "agpu_init_laser": (C.c_int, [_P, C.POINTER(AgpuLaser)]),
    "agpu_init_lp_fields": (C.c_int, [_P, C.POINTER(AgpuLpPulse)]),
    "agpu_envar_species": (C.c_int, [_P, C.c_int32, C.c_double, C.POINTER(AgpuEnvarOut)]),
    "agpu_envar_fields": (C.c_int, [_P, C.POINTER(AgpuEnvarFieldsOut)]),
    "agpu_set_ionization_table": (C.c_int, [_P, C.c_int32, _D, C.c_int32, C.c_int32, C.c_double]),
    "agpu_build_ionization_table": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, _D,
                                              C.POINTER(C.c_double)]),
    "agpu_set_ionization_species": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                              C.c_int32, C.c_double]),
    "agpu_step": (C.c_int, [_P, C.c_int32, C.c_double, C.c_int32, C.POINTER(AgpuStepOut)]),
    "agpu_window_inject": (C.c_int, [_P, C.c_int32, _D, C.c_int64, C.c_int64, C.c_int32]),
    "agpu_env_enable": (C.c_int, [_P, C.POINTER(AgpuEnvParams)]),
    "agpu_set_envelope": (C.c_int, [_P, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "agpu_get_envelope": (C.c_int, [_P, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "agpu_get_env_source": (C.c_int, [_P, _D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "agpu_init_envelope": (C.c_int, [_P, C.POINTER(AgpuLpPulse), C.c_int32]),
    "agpu_env_run": (C.c_int, [_P, C.c_int32, C.c_double, C.POINTER(AgpuStepOut)]),
    "agpu_beam_inject": (C.c_int, [_P, C.c_int32, _D, C.c_int64, C.c_int64, C.c_int32, C.c_double]),
    "agpu_beam_potential": (C.c_int, [_P, _D, _D, C.c_double]),
    "agpu_set_deferred_counts": (C.c_int, [_P, C.c_int32]),
    "agpu_set_step_graphs": (C.c_int, [_P, C.c_int32]),
    "agpu_set_fused_yee": (C.c_int, [_P, C.c_int32]),
    "agpu_batch_create": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    "agpu_batch_destroy": (C.c_int, [_P]),
    "agpu_batch_size": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "agpu_batch_handle": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    "agpu_batch_run": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "agpu_batch_set_graphs": (C.c_int, [_P, C.c_int32]),
    "agpu_batch_set_multi": (C.c_int, [_P, C.c_int32]),
    "agpu_batch_launches": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "agpu_batch_clock": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "agpu_diag": (C.c_int, [_P, C.POINTER(AgpuDiagOut)]),
    "agpu_set_profiling": (C.c_int, [_P, C.c_int32]),
    "agpu_get_timers": (C.c_int, [_P, C.POINTER(AgpuTimers)]),
    "agpu_reset_timers": (C.c_int, [_P]),
    "agpu_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "agpu_synchronize": (C.c_int, [_P]),
    "agpu_set_sort_interval": (C.c_int, [_P, C.c_int32]),
    "agpu_get_window_state": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_double)]),
    "agpu_set_window_state": (C.c_int, [_P, C.c_double, C.POINTER(C.c_int64)]),
    "agpu_set_deterministic": (C.c_int, [_P, C.c_int32]),
    "agpu_struct_sizes": (C.c_int, [C.POINTER(C.c_int64), C.c_int32]),
    "agpu_field_diag_noalloc": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                          C.c_double, _P, _P]),
    "agpu_set_stretch": (C.c_int, [_P, C.POINTER(AgpuStretch)]),
    "agpu_set_subdomain": (C.c_int, [_P, C.c_int32, C.c_int32, HALO_FN, _P]),
    "agpu_set_subdomain_yz": (C.c_int, [_P, C.POINTER(C.c_int32), HALO_FN, _P]),
    "agpu_halo_size_z": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    "agpu_halo_pack_z": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P]),
    "agpu_halo_unpack_z": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32]),
    "agpu_halo_size": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    "agpu_halo_pack": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P]),
    "agpu_halo_unpack": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32]),
    "agpu_halo_emigrants": (C.c_int, [_P, C.c_int32, C.c_int32, _P, C.c_int64, C.POINTER(C.c_int64)]),
    "agpu_halo_immigrants": (C.c_int, [_P, C.c_int32, _P, C.c_int64, C.c_int64]),
}

_lib = None


class AgpuError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = f"{where} failed with status {code}"
        if _lib is not None:
            try:
                msg += ": " + _lib.agpu_error_string(code).decode()
            except Exception:  # pragma: no cover - message only
                pass
        super().__init__(msg)
        self.code = code


def load_library(path: str | None = None):
    """Load the in-tree device library; raise if it has not been built.

    There is no CPU fallback: a missing library is an error.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"device library {p} is missing; build it with "
            "`python -m aladyn_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(code: int, where: str):
    if code != AGPU_OK:
        raise AgpuError(code, where)
