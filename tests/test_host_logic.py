"""Host-side checks of the index and binning helpers the device kernels use
(multiply-high cell decomposition, binning keys of tile, row and offset
octant): tests/host/host_logic.cu is compiled by nvcc into a temporary
directory and run on the CPU (it makes no CUDA call)."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not found")
def test_host_logic():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "host_logic")
        subprocess.run([NVCC, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "aladyn_b200", "csrc"),
                        "-gencode", "arch=compute_100a,code=sm_100a",
                        os.path.join(HERE, "host", "host_logic.cu"), "-o", exe],
                       check=True, capture_output=True, timeout=600)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.startswith("host logic ok")
