"""CPU checks of the C-ABI library and the host-side logic: the library loads
and exports every function the header declares, the struct layouts agree,
the host-only ADK table builder agrees with the oracle's bit for bit, the
host lattice generator with the oracle's loader, and the derived parameters
with the reference's formulas.  No device call is made."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from aladyn_b200 import abi
from aladyn_b200.abi import AgpuDiagOut, AgpuLaser, AgpuParams, AgpuPlasma, AgpuStepOut, AgpuTimers
from aladyn_b200.config import Grid, make_params, ompe_value
from aladyn_b200.lattice import LatticeHost, philox4x32_10
from oracle.oracle import NGE, Oracle, build_ionization_table
from tests.helpers import plasma_source, small_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aladyn_gpu.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(agpu_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_function():
    lib = abi.load_library()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
        assert n in abi.SIGNATURES, f"{n} missing from the ctypes mirror"


def test_struct_layouts_match():
    lib = abi.load_library()
    sizes = (C.c_int64 * 6)()
    assert lib.agpu_struct_sizes(sizes, 6) == 0
    for s, cls in zip(sizes, (AgpuParams, AgpuPlasma, AgpuLaser, AgpuStepOut, AgpuDiagOut, AgpuTimers)):
        assert s == C.sizeof(cls), cls.__name__


def test_create_fails_loudly_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = abi.load_library()
    p = small_case(2)
    h = C.c_void_p()
    assert lib.agpu_create(C.byref(p), C.byref(h)) == abi.AGPU_E_NODEVICE
    assert not h.value
    # a batch of instances reports the same, and creates nothing
    arr = (abi.AgpuParams * 3)(p, p, p)
    b = C.c_void_p()
    assert lib.agpu_batch_create(C.cast(arr, C.c_void_p), 3, C.byref(b)) == abi.AGPU_E_NODEVICE
    assert not b.value
    assert lib.agpu_batch_create(C.cast(arr, C.c_void_p), 0, C.byref(b)) == abi.AGPU_E_ARG


@pytest.mark.parametrize("an,z0,model", [(7, 0, 1), (7, 0, 4), (7, 2, 2), (2, 0, 3), (6, 0, 5), (1, 0, 1)])
def test_library_ionization_table_equals_oracle(an, z0, model):
    lib = abi.load_library()
    tab = np.zeros((NGE + 2, an + 1), order="F")
    de = C.c_double()
    rc = lib.agpu_build_ionization_table(an, z0, model, 2.7, 0.031, tab.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.byref(de))
    assert rc == 0
    ref, de_ref = build_ionization_table(an, z0, model, 2.7, 0.031)
    assert de.value == de_ref
    assert np.array_equal(tab.view(np.uint64), ref.view(np.uint64))


def test_host_philox_matches_published_vectors():
    r = philox4x32_10(np.array([0x243F6A88], np.uint32), np.array([0x85A308D3], np.uint32),
                      np.array([0x13198A2E], np.uint32), np.array([0x03707344], np.uint32), 0xA4093822, 0x299F31D0)
    assert [int(x[0]) for x in r] == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("ndim", [2, 3])
def test_host_lattice_equals_oracle_loader(ndim):
    p = small_case(ndim, nx=32, ny=16, nz=12, cap=50_000)
    src = plasma_source(p)
    o = Oracle(p)
    o.set_plasma_source(src)
    o.load_plasma(0)
    ref = o.get_species(0)
    host = LatticeHost(p, src)
    i2 = host.columns_end(1, p.xmax, False)
    rec = host.records(1, i2)
    assert rec.shape == ref.shape
    assert np.array_equal(rec.view(np.uint64), ref.view(np.uint64))


def test_derived_parameters_follow_the_reference():
    """dt, djc, ompe and the box bounds of set_initial_param / set_grid."""
    g = Grid(3, 1024, 256, 256, k0=25.0, yx_rat=5.0, zx_rat=5.0, cfl=0.8)
    p = make_params(g)
    dx = 1.0 / 25.0
    assert p.dx == dx and p.dy == 5.0 * dx and p.dz == 5.0 * dx
    assert p.dt == 0.8 / math.sqrt((1 / dx) ** 2 + (1 / p.dy) ** 2 + (1 / p.dz) ** 2)
    assert (p.djc[0], p.djc[1], p.djc[2]) == (dx / 3.0, p.dy / 3.0, p.dz / 3.0)
    assert p.gxmin == 0.0 and p.gxmax == 1024 * dx and p.xmax == 1023 * dx
    assert p.gymin == -128 * p.dy and p.gymax == 128 * p.dy
    assert abs(ompe_value() - 4 * math.pi * 2.81794033 * 1e-3) < 1e-15
    g2 = Grid(2, 1024, 256, 1, k0=25.0, yx_rat=4.0, zx_rat=1.0, cfl=0.8)
    p2 = make_params(g2)
    assert (p2.djc[0], p2.djc[1]) == (0.5 * dx, 0.5 * 4.0 * dx)
    assert p2.nfield == 3 and p2.curr_ndim == 2
