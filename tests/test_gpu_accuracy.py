"""Accuracy of the FP32 split form against the FP64 form over a long run:
the same seeded LWFA workload (laser, jittered lattice plasma, moving
window) advanced 1000 steps in both forms; the relative L2 difference of
every field component stays within 1e-3 (the split form's accuracy target),
and the particle counts agree to 0.1%."""
import math

import numpy as np
import pytest

import bench
from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload,steps", [("lwfa3d_128x64x64_ppc8", 1000), ("lwfa2d_1024x256_ppc4", 1000)])
def test_fp32_split_vs_fp64_long_run(workload, steps):
    res = {}
    for prec in (AGPU_FP64, AGPU_FP32_SPLIT):
        dev, p, las, src, ppc = bench.load_device(workload, prec, cap_factor=1.6)
        t = 0.0
        for it in range(steps):
            out = dev.lp_run(t, it, initial_time=(it == 0))
            assert out.error_bits == 0
            t += p.dt
        res[prec] = (dev.get_fields(), dev.count(0), p)
        dev.close()
    f64, n64, p = res[AGPU_FP64]
    f32, n32, _ = res[AGPU_FP32_SPLIT]
    err = bench.rel_l2_errors(f32, f64, p)
    print(workload, "rel L2 per component after", steps, "steps:", err, "counts", n32, n64)
    assert all(e <= 1e-3 for e in err), err
    assert abs(n32 - n64) <= 1e-3 * n64
