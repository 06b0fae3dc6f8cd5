"""The public header as a C host sees it: include/aladyn_gpu.h compiles as
strict C99 and as C++11 (the extern "C" guard), and a C program that takes
the address of every declared entry point links against libaladyn_gpu.so
(each declared name resolves in the library at link time) and runs the
host-only calls (struct sizes, error strings) without a device."""
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
