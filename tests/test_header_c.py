"""The public header as a C host sees it: include/aladyn_gpu.h compiles as
strict C99 and as C++11 (the extern "C" guard), and a C program that takes
the address of every declared entry point links against libaladyn_gpu.so
(each declared name resolves in the library at link time) and runs the
host-only calls (struct sizes, error strings) without a device; every
struct member's offset as a C compiler lays it out equals the ctypes
mirror's."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from aladyn_b200 import abi
from aladyn_b200.abi import AgpuDiagOut, AgpuLaser, AgpuParams, AgpuPlasma, AgpuStepOut, AgpuTimers
from tests.test_abi import HEADER, ROOT, header_functions

CC = shutil.which("gcc")
CXX = shutil.which("g++")


def _program(names):
    refs = ",\n  ".join(f"(fn_t){n}" for n in names)
    return f"""#include <stdio.h>
#include <string.h>
#include "aladyn_gpu.h"
typedef void (*fn_t)(void);
static const fn_t entry_points[] = {{
  {refs}
}};
int main(void) {{
  int64_t sizes[6];
  int i;
  for (i = 0; i < (int)(sizeof entry_points / sizeof entry_points[0]); ++i)
    if (!entry_points[i]) return 3;
  if (agpu_struct_sizes(sizes, 6) != 0) return 4;
  for (i = 0; i < 6; ++i) printf("%lld\\n", (long long)sizes[i]);
  if (!agpu_error_string(0) || strlen(agpu_error_string(0)) == 0) return 5;
  printf("%d\\n", (int)(sizeof entry_points / sizeof entry_points[0]));
  return 0;
}}
"""


@pytest.mark.skipif(CC is None or CXX is None, reason="needs gcc and g++")
def test_header_compiles_and_links_from_c(tmp_path):
    lib = abi.load_library()
    so = lib._name
    names = header_functions()
    src = tmp_path / "host.c"
    src.write_text(_program(names))
    inc = os.path.dirname(HEADER)
    exe = tmp_path / "host"
    # pedantic C99: function-pointer casts between function types are allowed
    subprocess.run([CC, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", inc, str(src),
                    "-o", str(exe), so, f"-Wl,-rpath,{os.path.dirname(so)}"], check=True, cwd=ROOT)
    subprocess.run([CXX, "-std=c++11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-x", "c++", "-I", inc,
                    "-fsyntax-only", str(src)], check=True, cwd=ROOT)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    structs = (AgpuParams, AgpuPlasma, AgpuLaser, AgpuStepOut, AgpuDiagOut, AgpuTimers)
    assert [int(v) for v in out[:6]] == [C.sizeof(c) for c in structs]
    assert int(out[6]) == len(names)


STRUCTS = {
    "agpu_params": "AgpuParams", "agpu_plasma": "AgpuPlasma", "agpu_laser": "AgpuLaser",
    "agpu_lp_pulse": "AgpuLpPulse", "agpu_step_out": "AgpuStepOut", "agpu_diag_out": "AgpuDiagOut",
    "agpu_timers": "AgpuTimers", "agpu_env_params": "AgpuEnvParams", "agpu_envar_out": "AgpuEnvarOut",
    "agpu_envar_fields_out": "AgpuEnvarFieldsOut", "agpu_stretch_axis": "AgpuStretchAxis",
    "agpu_stretch": "AgpuStretch",
}


@pytest.mark.skipif(CC is None, reason="needs gcc")
def test_every_struct_field_offset_matches_the_ctypes_mirror(tmp_path):
    """offsetof and sizeof of every member of every struct the header
    declares, as a C compiler lays them out, equal the ctypes mirror's
    (same member names: a renamed or reordered member fails to compile or
    to match)."""
    lines, want = [], []
    for cname, pyname in STRUCTS.items():
        cls = getattr(abi, pyname)
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        want.append(C.sizeof(cls))
        for fname, _ in cls._fields_:
            if fname.startswith("reserved"):
                continue
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
            want.append(getattr(cls, fname).offset)
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"aladyn_gpu.h\"\nint main(void) {\n"
                   + "\n".join(lines) + "\n  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([CC, "-std=c99", "-Wall", "-Werror", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                   check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == want
    assert len(want) > 100
