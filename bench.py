#!/usr/bin/env python
"""Benchmark of the B200 PIC step: particle-pushes/s of the 3D LWFA step
(1024x256x256 cells, 8 particles/cell, ~5.4e8 electrons, moving window) in the
FP32 split form and the plain FP64 form on one GPU, plus the Yee update GB/s.

Contract (one JSON line from rank 0):
  value      whole-job particle-pushes/s of the FP32 split form: particles x
             steps / device time of the full step (gather, push, deposit,
             box-edge removal, current fold, Yee update, window shift);
  e2e        the same metric through the C-ABI with host buffers: every step
             the host's window-injection records are copied from pinned host
             memory (agpu_window_inject) and the step output plus the FP64
             diagnostics come back (agpu_step, agpu_diag);
  roofline   the fused gather+push+deposit kernel of the FP32 split form
             against the measured HBM copy bandwidth;
  cpu_baseline the oracle (CPU FP64 restatement of the reference) on all
             host cores on a bounded sample of the same workload.

--impl reference times the oracle alone (the reference's CPU arithmetic) on
the host cores.  Under torchrun (N > 1) every rank runs one independent
replica of the workload on its own GPU (replicas only: no collective on the
data path) and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

LAM0 = 0.8  # um

# Workloads (the reference's LWFA setups restated on synthetic seeded input)
WORKLOADS = {
    # 3D LWFA: 1024x256x256, dx = 0.05 lambda, dy = dz = 0.25 lambda, 8 ppc,
    # n_e = 0.005 n_c, a0 = 3, waist 6 lambda, FWHM 10 lambda/c, window at c.
    "lwfa3d_1024x256x256_ppc8": dict(ndim=3, nx=1024, ny=256, nz=256, k0=25.0, yx_rat=5.0, zx_rat=5.0,
                                    cfl=0.8, ppc=(2, 2, 2), n_over_nc=0.005, a0=3.0, w0=6 * LAM0,
                                    tau=10 * LAM0, x_plasma=0.0, xc_frac=0.7),
    # 2D LWFA: 1024x256, dx = 0.05 lambda, dy = 0.2 lambda, 4 ppc, n_e = 0.01 n_c,
    # plasma from x = 20 lambda, a0 = 2, waist 5 lambda.
    "lwfa2d_1024x256_ppc4": dict(ndim=2, nx=1024, ny=256, nz=1, k0=25.0, yx_rat=4.0, zx_rat=1.0,
                                 cfl=0.8, ppc=(2, 2, 1), n_over_nc=0.01, a0=2.0, w0=5 * LAM0,
                                 tau=10 * LAM0, x_plasma=20 * LAM0, xc_frac=0.3),
    # the same 3D workload with the cubic shape extension (the reference
    # gathers and deposits with quadratic shapes only)
    "lwfa3d_1024x256x256_ppc8_cubic": dict(ndim=3, nx=1024, ny=256, nz=256, k0=25.0, yx_rat=5.0, zx_rat=5.0,
                                          cfl=0.8, ppc=(2, 2, 2), n_over_nc=0.005, a0=3.0, w0=6 * LAM0,
                                          tau=10 * LAM0, x_plasma=0.0, xc_frac=0.7, shape=1),
    # small 3D cases for quick checks and profiler captures
    "lwfa3d_128x64x64_ppc8": dict(ndim=3, nx=128, ny=64, nz=64, k0=25.0, yx_rat=5.0, zx_rat=5.0,
                                 cfl=0.8, ppc=(2, 2, 2), n_over_nc=0.005, a0=3.0, w0=6 * LAM0,
                                 tau=10 * LAM0, x_plasma=0.0, xc_frac=0.7),
    "lwfa3d_256x128x128_ppc8": dict(ndim=3, nx=256, ny=128, nz=128, k0=25.0, yx_rat=5.0, zx_rat=5.0,
                                   cfl=0.8, ppc=(2, 2, 2), n_over_nc=0.005, a0=3.0, w0=6 * LAM0,
                                   tau=10 * LAM0, x_plasma=0.0, xc_frac=0.7),
    # the physical box of lwfa3d_1024x256x256_ppc8 at 3/8 of its resolution:
    # the same laser-to-box volume fraction with 28e6 particles (profiler
    # captures of the kernel mix the full-size step sees)
    "lwfa3d_384x96x96_ppc8": dict(ndim=3, nx=384, ny=96, nz=96, k0=9.375, yx_rat=5.0, zx_rat=5.0,
                                 cfl=0.8, ppc=(2, 2, 2), n_over_nc=0.005, a0=3.0, w0=6 * LAM0,
                                 tau=10 * LAM0, x_plasma=0.0, xc_frac=0.7),
}
DEFAULT_WORKLOAD = "lwfa3d_1024x256x256_ppc8"

# Batched 2D scan: 256 LWFA instances, nx in {256..1024} x ny in {64, 128, 256}
# (dx = 0.05 lambda, dy = 0.2 lambda, 4 ppc), a0 ~ U[1, 4], waist ~ U[3, 8]
# lambda, n_e/n_c ~ logU[0.002, 0.02], drawn with Philox(seed, instance).
SCAN_WORKLOAD = "scan2d_256"
SCAN_NX = (256, 384, 512, 768, 1024)
SCAN_NY = (64, 128, 256)


def scan_instances(n: int, precision: int, seed: int = 20241205):
    from aladyn_b200.config import Grid, laser, make_params, n_over_nc_to_n0, plasma
    from aladyn_b200.lattice import philox4x32_10
    idx = np.arange(n, dtype=np.uint32)
    z = np.zeros(n, dtype=np.uint32)
    r = philox4x32_10(idx, z, z, np.full(n, 0x5343414E, dtype=np.uint32), seed, 0)
    r2 = philox4x32_10(idx, z, z + 1, np.full(n, 0x5343414E, dtype=np.uint32), seed, 0)
    u = [(x.astype(np.float64) + 0.5) / 4294967296.0 for x in (*r, *r2)]
    out = []
    for i in range(n):
        nx = SCAN_NX[int(u[0][i] * len(SCAN_NX))]
        ny = SCAN_NY[int(u[1][i] * len(SCAN_NY))]
        a0 = 1.0 + 3.0 * u[2][i]
        w0 = (3.0 + 5.0 * u[3][i]) * LAM0
        n_over_nc = 10.0 ** (math.log10(0.002) + u[4][i] * (math.log10(0.02) - math.log10(0.002)))
        g = Grid(2, nx, ny, 1, 25.0, 4.0, 1.0, 0.8)
        cap = int(nx * ny * 4 * 1.04) + 4096
        p = make_params(g, precision=precision, capacity=(cap, 0, 0, 0), w_sh=10, w_speed=1.0)
        lx = nx * p.dx
        las = laser(a0, LAM0, w0, 10 * LAM0, xc=0.5 * lx, xf=0.5 * lx)
        n0 = n_over_nc_to_n0(n_over_nc, LAM0)
        src = plasma(0, 2, 2, 1, -1, n0 / 4, x_start=p.gxmin, x_end=1.0e7, y_min=p.gymin, y_max=p.gymax,
                     jitter=0.5, seed=seed + i)
        out.append((p, las, src))
    return out


def bytes_per_push(ndim: int, ppc: int, fp32: bool) -> float:
    """Algorithmic bytes of one particle push (gather+push+deposit):
    particle record read + written once, fields read and currents written
    once per cell, amortised over the particles of a cell.
    FP64 3D: read x,p,w 56 B + write x,p 48 B + (6 field + 3 current words) x 8 B / ppc.
    FP32 split 3D: read node 4 + offsets 12 + p 12 + slot 8 B, write node,
    offsets, p 28 B, fields 24 B + currents (hi, lo) 24 B per cell / ppc."""
    if ndim == 3:
        return (36.0 + 28.0 + 48.0 / ppc) if fp32 else (104.0 + 72.0 / ppc)
    return (24.0 + 20.0 + 28.0 / ppc) if fp32 else (72.0 + 40.0 / ppc)


# DRAM bytes (read + write) per particle of one k32_tile launch, from an ncu
# capture of the 384x96x96-cell, 8 ppc workload two steps after a window
# shift (2045.8 MB for 2.83e7 particles); traffic grows in proportion to the
# particles of a launch.
K32_DRAM_BYTES_PER_PUSH = 72.3


def yee_bytes_per_cell(ndim: int, fp32: bool) -> float:
    """Read E, B, J and write E, B once: 15 words (3D) or 8 words (2D TE)."""
    return (15 if ndim == 3 else 8) * (4 if fp32 else 8)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# workload set-up on the device
# --------------------------------------------------------------------------
def make_workload(name: str, precision: int, cap_factor: float = 1.04):
    from aladyn_b200.config import Grid, laser, make_params, n_over_nc_to_n0, plasma
    w = WORKLOADS[name]
    g = Grid(w["ndim"], w["nx"], w["ny"], w["nz"], w["k0"], w["yx_rat"], w["zx_rat"], w["cfl"])
    ppc = w["ppc"][0] * w["ppc"][1] * (w["ppc"][2] if w["ndim"] == 3 else 1)
    ncell = w["nx"] * w["ny"] * (w["nz"] if w["ndim"] == 3 else 1)
    cap = int(ncell * ppc * cap_factor) + 4096
    p = make_params(g, precision=precision, capacity=(cap, 0, 0, 0), w_sh=10, w_speed=1.0, shape=w.get("shape", 0))
    lx = w["nx"] * p.dx
    las = laser(w["a0"], LAM0, w["w0"], w["tau"], xc=w["xc_frac"] * lx, xf=w["xc_frac"] * lx)
    n0 = n_over_nc_to_n0(w["n_over_nc"], LAM0)
    src = plasma(0, w["ppc"][0], w["ppc"][1], w["ppc"][2] if w["ndim"] == 3 else 1, -1, n0 / ppc,
                 x_start=p.gxmin + w["x_plasma"], x_end=1.0e7, y_min=p.gymin, y_max=p.gymax,
                 z_min=p.gzmin, z_max=p.gzmax, jitter=0.5, seed=20241203)
    return p, las, src, ppc


def load_device(name, precision, host_injection=False, cap_factor=1.04):
    """The workload on a fresh device handle.  cap_factor sizes the particle
    capacity over cells x ppc: long runs need headroom, the laser pushes
    electrons forward while the window keeps injecting fresh columns."""
    from aladyn_b200.sim import PicDevice
    p, las, src, ppc = make_workload(name, precision, cap_factor)
    dev = PicDevice(p)
    dev.init_laser(las)
    if host_injection:
        # the device loads the initial columns; later columns come from the host
        from aladyn_b200.config import plasma
        s2 = plasma(src.ic, src.npx, src.npy, src.npz, src.charge, src.wgh, x_start=src.x_start,
                    x_end=p.xmax + 1e-9, y_min=src.y_min, y_max=src.y_max, z_min=src.z_min,
                    z_max=src.z_max, jitter=src.jitter, seed=src.seed)
        dev.set_plasma_source(s2)
    else:
        dev.set_plasma_source(src)
    dev.load_plasma(0)
    return dev, p, las, src, ppc


def rel_l2_errors(fa, fb, p):
    sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2) if p.ndim == 3 else slice(0, 1))
    out = []
    for c in range(p.nfield):
        a, b = fa[sl + (c,)], fb[sl + (c,)]
        nb = float(np.linalg.norm(b))
        out.append(float(np.linalg.norm(a - b)) / nb if nb > 0 else 0.0)
    return out


def timed_steps(dev, p, t, it, k, torch):
    """Run k steps; device time by CUDA events on the library's stream."""
    s = torch.cuda.ExternalStream(dev.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev.synchronize()
    e0.record(s)
    nsum = 0
    for _ in range(k):
        out = dev.lp_run(t, it, initial_time=(it == 0))
        nsum += out.np[0] + out.removed[0] - out.injected[0]  # particles pushed this step
        t += p.dt
        it += 1
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1), nsum, t, it, out


def run_form(name, precision, warmup, steps, torch, barrier, keep_fields=False, graphs=False):
    """Warm-up, then the timed region with profiling timers on.  graphs:
    deferred counts and step graphs (the library's fastest form of a step
    on small grids, where launches dominate); the pushes then come from the
    library's own counters."""
    dev, p, las, src, ppc = load_device(name, precision)
    if graphs:
        dev.set_deferred_counts(True)
        dev.set_step_graphs(True)
    t, it = 0.0, 0
    for _ in range(warmup):
        dev.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
        it += 1
    dev.set_profiling(True)
    dev.reset_timers()
    barrier()
    ms, pushes, t, it, out = timed_steps(dev, p, t, it, steps, torch)
    if graphs:
        dev.set_deferred_counts(False)  # synchronises and refreshes the counters
        pushes = dev.timers().pushes
    tm = dev.timers()
    fields = dev.get_fields() if keep_fields else None
    res = dict(ms=ms, pushes=pushes, np=out.np[0], err=out.error_bits, timers=tm, p=p, ppc=ppc,
               fields=fields, steps=steps)
    dev.close()
    return res


def run_e2e(name, precision, warmup, steps, torch, barrier):
    """Through the C-ABI with host buffers: the host supplies the window
    injection records from pinned memory and reads the step output and the
    FP64 diagnostics every step."""
    from aladyn_b200.lattice import LatticeHost
    dev, p, las, src, ppc = load_device(name, precision, host_injection=True)
    host = LatticeHost(p, src)
    host.nptx = host.columns_end(1, p.xmax, False)
    # window schedule of lp_window_xshift (window.f90:276-347), replayed on
    # the host to prepare every step's injection records before timing
    total = warmup + steps
    xlapse, wi1, xmax = 0.0, 0, p.xmax
    inject = {}
    for it in range(total):
        tt = it * p.dt  # only the wi/wf window bounds use t; they are open here
        if p.w_sh > 0 and it % p.w_sh == 0 and p.wi_time <= tt < p.wf_time:
            if it == 0:
                xlapse, wi1 = 0.0, 0
                continue
            xlapse = xlapse + p.w_speed * p.dt * float(p.w_sh)
            wi2 = int(math.floor(abs(p.dx_inv * xlapse) + 0.5))
            nshx = wi2 - wi1
            wi1 = wi2
            xmax = xmax + p.dx * float(nshx)
            rec = host.inject_after_shift(xmax)
            if rec.shape[0] > 0:
                buf = torch.empty(rec.shape[::-1], dtype=torch.float64, pin_memory=True).numpy().T
                buf[...] = rec
                inject[it] = buf
    t, it = 0.0, 0
    h2d = 0
    nsum = 0
    for phase, k in (("warm", warmup), ("timed", steps)):
        if phase == "timed":
            barrier()
            s = torch.cuda.ExternalStream(dev.stream())
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            dev.synchronize()
            e0.record(s)
        for _ in range(k):
            out = dev.lp_run(t, it, initial_time=(it == 0))
            if phase == "timed":
                nsum += out.np[0] + out.removed[0] - out.injected[0]
            if it in inject:
                dev.window_inject(0, inject[it])
                if phase == "timed":
                    h2d += inject[it].nbytes
            dev.diag()
            t += p.dt
            it += 1
        if phase == "timed":
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
    from aladyn_b200.abi import AgpuDiagOut, AgpuStepOut
    d2h = steps * (C.sizeof(AgpuStepOut) + C.sizeof(AgpuDiagOut))
    dev.close()
    return dict(ms=ms, pushes=nsum, h2d=h2d / steps, d2h=d2h / steps)


# --------------------------------------------------------------------------
# CPU: the oracle (FP64 restatement of the reference's arithmetic)
# --------------------------------------------------------------------------
def cpu_sample(name, budget_s=15.0, threads=None, warmup=0, steps=None):
    """The oracle on a bounded sample of the workload: the same cell size,
    time step, plasma and laser on a sub-box with the same particles per cell
    (the transverse and longitudinal extent reduced), stepped for about
    budget_s seconds on all host cores."""
    from aladyn_b200.abi import AGPU_FP64
    from aladyn_b200.config import Grid, laser, make_params, n_over_nc_to_n0, plasma
    from aladyn_b200.initial import laser_fields
    from oracle.oracle import Oracle
    w = dict(WORKLOADS[name])
    if w["ndim"] == 3:
        w.update(nx=256, ny=64, nz=64)
    else:
        w.update(nx=512, ny=128)
    threads = threads or os.cpu_count() or 1
    g = Grid(w["ndim"], w["nx"], w["ny"], w["nz"], w["k0"], w["yx_rat"], w["zx_rat"], w["cfl"])
    ppc = w["ppc"][0] * w["ppc"][1] * (w["ppc"][2] if w["ndim"] == 3 else 1)
    ncell = w["nx"] * w["ny"] * (w["nz"] if w["ndim"] == 3 else 1)
    p = make_params(g, precision=AGPU_FP64, capacity=(int(ncell * ppc * 1.1) + 4096, 0, 0, 0), w_sh=10)
    lx = w["nx"] * p.dx
    las = laser(w["a0"], LAM0, min(w["w0"], 0.25 * w["ny"] * p.dy), w["tau"], xc=w["xc_frac"] * lx,
                xf=w["xc_frac"] * lx)
    n0 = n_over_nc_to_n0(w["n_over_nc"], LAM0)
    src = plasma(0, w["ppc"][0], w["ppc"][1], w["ppc"][2] if w["ndim"] == 3 else 1, -1, n0 / ppc,
                 x_start=p.gxmin + min(w["x_plasma"], 0.2 * lx), x_end=1.0e7, y_min=p.gymin, y_max=p.gymax,
                 z_min=p.gzmin, z_max=p.gzmax, jitter=0.5, seed=20241203)
    ora = Oracle(p, threads=threads)
    ora.set_fields(laser_fields(p, las))
    ora.set_plasma_source(src)
    ora.load_plasma(0)
    t, it, pushes = 0.0, 0, 0
    for _ in range(warmup):
        ora.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
        it += 1
    t0 = time.perf_counter()
    done = 0
    while True:
        n = ora.count(0)
        rc, out = ora.lp_run(t, it, initial_time=(it == 0))
        pushes += n
        t += p.dt
        it += 1
        done += 1
        el = time.perf_counter() - t0
        if steps is not None:
            if done >= steps:
                break
        elif el >= budget_s or done >= 200:
            break
    sample = (f"{w['nx']}x{w['ny']}" + (f"x{w['nz']}" if w["ndim"] == 3 else "") +
              f" cells, {ppc} ppc, {n} particles, {done} timed steps after {warmup} warm-up, "
              f"FP64 oracle on {threads} threads")
    return dict(value=pushes / el, cores=threads, sample=sample, steps=done, seconds=el)


def make_reducers(torch, world: int, device: str):
    """Barrier and max/sum over ranks for the replicas-only multi-GPU run
    (timing is the max over ranks, work the sum); identity at one rank."""
    if world <= 1:
        def barrier():
            if device == "cuda":
                torch.cuda.synchronize()

        return barrier, (lambda x: x), (lambda x: x)
    import torch.distributed as dist

    def barrier():
        dist.barrier()
        if device == "cuda":
            torch.cuda.synchronize()

    def red(x, op):
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    return barrier, (lambda x: red(x, dist.ReduceOp.MAX)), (lambda x: red(x, dist.ReduceOp.SUM))


def scan_measure(torch, warmup, steps, threads=0, n=256, sort_interval=0):
    """Batched scan: the n instances advanced together (agpu_batch_run)
    against the same instances run one after the other through the
    single-instance path in its fastest form (deferred counts, each step
    replayed from its captured CUDA graph), so that the ratio measures the
    batching, not removed host synchronisations.  Both arms: fresh
    instances, W warm-up steps, then K timed steps; device time by CUDA
    events bracketing the timed steps after a synchronisation."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT
    from aladyn_b200.sim import PicBatch, PicDevice
    cases = scan_instances(n, AGPU_FP32_SPLIT)
    for p, _, _ in cases:  # headroom: the lasers push electrons forward as the window injects
        p.capacity[0] = int(p.capacity[0] * 1.5)

    def setup(d, las, src):
        d.init_laser(las)
        d.set_plasma_source(src)
        d.load_plasma(0)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # batched arm
    batch = PicBatch([c[0] for c in cases])
    for d, (p, las, src) in zip(batch.instances, cases):
        setup(d, las, src)
        d.set_sort_interval(sort_interval)
    st = batch.run(warmup, threads)
    if st != [0] * n:
        raise RuntimeError(f"batched warm-up failed: {st}")
    for d in batch.instances:
        d.reset_timers()
    launches0 = batch.launches()
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record()
    st = batch.run(steps, threads)
    e1.record()
    e1.synchronize()
    ms_b = e0.elapsed_time(e1)
    if st != [0] * n:
        raise RuntimeError(f"batched steps failed: {st}")
    tms = [d.timers() for d in batch.instances]
    pushes_b = sum(t.pushes for t in tms)
    launches_b = sum(t.launches_total for t in tms) + batch.launches() - launches0
    batch.close()
    # sequential arm: one instance at a time, deferred counts + step graphs
    ms_s, pushes_s = 0.0, 0
    for (p, las, src) in cases:
        dev = PicDevice(p)
        setup(dev, las, src)
        dev.set_deferred_counts(True)
        dev.set_step_graphs(True)
        t, it = 0.0, 0
        for _ in range(warmup):
            dev.lp_run(t, it, initial_time=(it == 0))
            t += p.dt
            it += 1
        dev.synchronize()
        dev.reset_timers()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(steps):
            dev.lp_run(t, it, initial_time=(it == 0))
            t += p.dt
            it += 1
        dev.synchronize()
        e1.record()
        e1.synchronize()
        ms_s += e0.elapsed_time(e1)
        dev.set_deferred_counts(False)  # refreshes the push count on the host
        pushes_s += dev.timers().pushes
        dev.close()
    cells = sum(c[0].nx * c[0].ny for c in cases)
    return dict(ms_b=ms_b, ms_s=ms_s, pushes_b=pushes_b, pushes_s=pushes_s, launches_b=launches_b, cells=cells,
                value=n * steps / (ms_b * 1e-3), sequential=n * steps / (ms_s * 1e-3), n=n)


# --------------------------------------------------------------------------
# the other configurations, measured beside the headline workload
# --------------------------------------------------------------------------
def _guard(fn, *args):
    """One extra measurement; a failure is reported in its key instead of
    losing the line."""
    try:
        return fn(*args)
    except Exception as e:  # noqa: BLE001
        return {"error": f"{type(e).__name__}: {e}"}


def extra_forms(name, torch, warmup, steps, graphs=False):
    """Both precision forms of a workload: pushes/s of the full step, the
    push/deposit kernel's algorithmic GB/s and the Yee phase GB/s."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
    w = WORKLOADS[name]
    ppc = w["ppc"][0] * w["ppc"][1] * (w["ppc"][2] if w["ndim"] == 3 else 1)
    out = {"workload": name, "warmup": warmup, "steps": steps,
           "path": "deferred counts + step graphs" if graphs else "agpu_step, counts every step"}
    for key, prec in (("fp32_split", AGPU_FP32_SPLIT), ("fp64", AGPU_FP64)):
        r = run_form(name, prec, warmup, steps, torch, lambda: torch.cuda.synchronize(), graphs=graphs)
        tm, p = r["timers"], r["p"]
        cells = p.nx * p.ny * (p.nz if p.ndim == 3 else 1)
        fp32 = prec == AGPU_FP32_SPLIT
        out[key] = {"pushes_per_s": r["pushes"] / (r["ms"] * 1e-3), "ms_per_step": r["ms"] / steps,
                    "push_deposit_gbs": bytes_per_push(w["ndim"], ppc, fp32) * tm.pushes /
                    (tm.ms_push_deposit * 1e-3) / 1e9 if tm.ms_push_deposit else None,
                    "yee_gbs": yee_bytes_per_cell(p.ndim, fp32) * cells * steps / (tm.ms_yee * 1e-3) / 1e9
                    if tm.ms_yee else None,
                    "error_bits": r["err"]}
    out["fp32_over_fp64"] = out["fp32_split"]["pushes_per_s"] / out["fp64"]["pushes_per_s"]
    return out


def extra_c1(torch, warmup, steps):
    """C1 (2D, 1024x256, 4 ppc): both forms on the fixed path (deferred
    counts + step graphs), then the split form with the options the tuner
    (aladyn_b200/autotune.py) picks for this workload: sort interval, fused
    Yee, step graphs, each candidate timed on a fresh instance."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT
    from aladyn_b200.autotune import Tuner, tune_single
    name = "lwfa2d_1024x256_ppc4"
    out = extra_forms(name, torch, warmup, steps, True)
    p, _, _, ppc = make_workload(name, AGPU_FP32_SPLIT, 1.04)
    np0 = [0]

    def make():
        d = load_device(name, AGPU_FP32_SPLIT)[0]
        np0[0] = d.count(0)
        return d

    r = tune_single(torch, make, p, ppc, warmup, steps, tuner=Tuner(None))
    out["fp32_split_tuned"] = dict(r.as_dict(), pushes_per_s=np0[0] / (r.ms_per_step * 1e-3),
                                   note="particles at the start / tuned ms per step")
    return out


def extra_ionization(torch, warmup, steps):
    """3D ionization-injection LWFA (768x192x192, dx = 0.05 lambda, dy = dz =
    0.25 lambda): pre-ionised electrons at n_e = 0.005 n_c plus a 1%
    nitrogen dopant of neutral atoms (7 levels, one-level ADK model 1,
    Philox draws), 4 particles per cell each, laser a0 = 1.8, waist 6
    lambda, FWHM 10 lambda/c focused in the plasma.  Both forms: pushes/s
    (electrons) and the electrons born during the timed steps."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
    from aladyn_b200.config import Grid, laser, make_params, n_over_nc_to_n0, plasma
    from aladyn_b200.sim import PicDevice
    nx, ny, nz, a0 = 768, 192, 192, 1.8
    g = Grid(3, nx, ny, nz, 25.0, 5.0, 5.0, 0.8)
    ncell = nx * ny * nz
    n0 = n_over_nc_to_n0(0.005, LAM0)
    lp_max = 1.5 * a0 * 2.0 * math.pi / LAM0
    out = {"grid": [nx, ny, nz], "ppc_each": 4, "dopant": "N, 1% of n_e, 7 levels, ADK model 1",
           "warmup": warmup, "steps": steps}
    for key, prec in (("fp32_split", AGPU_FP32_SPLIT), ("fp64", AGPU_FP64)):
        p = make_params(g, precision=prec, nsp=2, nsp_run=1, capacity=(int(ncell * 4 * 1.5), int(ncell * 4 * 1.04), 0, 0),
                        w_sh=10, ionz_lev=1, n_mol_atoms=(1, 1, 1, 1), mass_number=(14.0, 1.0, 1.0))
        lx = nx * p.dx
        dev = PicDevice(p)
        dev.init_laser(laser(a0, LAM0, 6 * LAM0, 10 * LAM0, xc=0.6 * lx, xf=0.6 * lx))
        x0 = p.gxmin + 0.3 * lx
        dev.set_plasma_source(plasma(0, 2, 2, 1, -1, n0 / 4, x_start=x0, x_end=1.0e7, y_min=p.gymin,
                                     y_max=p.gymax, z_min=p.gzmin, z_max=p.gzmax, jitter=0.5, seed=20241204))
        dev.set_plasma_source(plasma(1, 2, 2, 1, 0, 0.01 * n0 / 4, x_start=x0, x_end=1.0e7, y_min=p.gymin,
                                     y_max=p.gymax, z_min=p.gzmin, z_max=p.gzmax, jitter=0.5, seed=20241205))
        dev.load_plasma(0)
        dev.load_plasma(1)
        dev.set_ionization_species(1, 7, 0, 7, 1, lp_max)
        t, it = 0.0, 0
        for _ in range(warmup):
            dev.lp_run(t, it, initial_time=(it == 0))
            t += p.dt
            it += 1
        dev.set_profiling(True)
        dev.reset_timers()
        s = torch.cuda.ExternalStream(dev.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dev.synchronize()
        e0.record(s)
        born, pushed, err = 0, 0, 0
        for _ in range(steps):
            o = dev.lp_run(t, it)
            born += o.new_electrons
            pushed += o.np[0] + o.removed[0] - o.injected[0] - o.new_electrons
            err |= o.error_bits
            t += p.dt
            it += 1
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        tm = dev.timers()
        out[key] = {"electron_pushes_per_s": pushed / (ms * 1e-3), "ms_per_step": ms / steps,
                    "ionize_ms_per_step": tm.ms_ionize / steps, "electrons_born": int(born),
                    "electrons": int(dev.count(0)), "ions": int(dev.count(1)), "error_bits": int(err)}
        dev.close()
    b32, b64 = out["fp32_split"]["electrons_born"], out["fp64"]["electrons_born"]
    out["born_fp32_over_fp64"] = b32 / b64 if b64 else None
    out["fp32_over_fp64"] = out["fp32_split"]["electron_pushes_per_s"] / out["fp64"]["electron_pushes_per_s"]
    return out


def extra_pwfa(torch, warmup, steps):
    """3D beam-driven PWFA, FP32 split form: 512x256x256 cells, dx = 0.2 um,
    dy = dz = 0.5 um, plasma n_e = 1e17 cm^-3 at 4 particles per cell, a
    bi-Gaussian driver of 2e7 macroparticles (200 pC, gamma 1957, 1% rms
    energy spread, sigma_z = 5 um, sigma_r = 3 um, 1 mm mrad); the bunch
    set-up (charge deposit and the FP64 sine-transform Poisson solve of its
    self-fields, agpu_beam_inject) timed once, then the standard cycle."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT
    from aladyn_b200.beam import Bunch, bunch_records
    from aladyn_b200.config import Grid, make_params, plasma
    from aladyn_b200.sim import PicDevice
    nx, ny, nz, nb = 512, 256, 256, 20_000_000
    g = Grid(3, nx, ny, nz, 5.0, 2.5, 2.5, 0.8)
    ncell = nx * ny * nz
    p = make_params(g, precision=AGPU_FP32_SPLIT, capacity=(int(ncell * 4 * 1.04) + nb + 4096, 0, 0, 0), w_sh=10)
    lx = nx * p.dx
    b = Bunch(nb_tot=nb, charge_pc=200.0, sxb=5.0, syb=3.0, gam=1957.0, epsy=1.0, epsz=1.0, dg=1.0,
              xc=p.xmn + 0.6 * lx, seed=77)
    t0 = time.perf_counter()
    rec = bunch_records(p, b, n0_ref=0.1)
    gen_s = time.perf_counter() - t0
    dev = PicDevice(p)
    dev.set_plasma_source(plasma(0, 2, 2, 1, -1, 0.25, x_start=p.gxmin, x_end=1.0e7, y_min=p.gymin, y_max=p.gymax,
                                 z_min=p.gzmin, z_max=p.gzmax, jitter=0.5, seed=20241206))
    dev.load_plasma(0)
    dev.synchronize()
    t0 = time.perf_counter()
    rc = dev.beam_inject(0, rec, b.gam)
    dev.synchronize()
    setup_s = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"agpu_beam_inject returned {rc}")
    n = dev.count(0)
    t, it = 0.0, 0
    for _ in range(warmup):
        dev.lp_run(t, it, initial_time=(it == 0))
        t += p.dt
        it += 1
    dev.set_profiling(True)
    dev.reset_timers()
    ms, pushes, t, it, o = timed_steps(dev, p, t, it, steps, torch)
    tm = dev.timers()
    dev.close()
    return {"grid": [nx, ny, nz], "bunch_macroparticles": nb, "particles": int(n), "form": "fp32_split",
            "bunch_setup_s": setup_s, "bunch_records_host_s": gen_s,
            "setup_note": "agpu_beam_inject wall time: record upload, charge deposit, FP64 DST-I Poisson "
                          "solve (cuFFT), bunch fields",
            "pushes_per_s": pushes / (ms * 1e-3), "ms_per_step": ms / steps,
            "push_deposit_ms_per_step": tm.ms_push_deposit / steps, "warmup": warmup, "steps": steps,
            "error_bits": int(o.error_bits)}


def extra_pwfa_envelope(torch, warmup, steps, nx=512, ny=256, nz=256, nb=20_000_000):
    """The reference's own PWFA route (Env_cycle: beam_inject, then env_run
    every step; model_id = 4 with a0 = 0 as its PWFA example): FP64 form,
    the 512x256x256 PWFA box and bunch of ``extra_pwfa``, der_ord 2, the
    envelope solver running on a zero envelope, plasma electrons and bunch
    in species 0 pushed by the envelope pusher."""
    from aladyn_b200.abi import AGPU_FP64
    from aladyn_b200.beam import Bunch, bunch_records
    from aladyn_b200.config import Grid, env_params, make_params, plasma
    from aladyn_b200.sim import PicDevice
    g = Grid(3, nx, ny, nz, 5.0, 2.5, 2.5, 0.8)
    ncell = nx * ny * nz
    p = make_params(g, precision=AGPU_FP64, capacity=(int(ncell * 4 * 1.04) + nb + 4096, 0, 0, 0), w_sh=10)
    lx = nx * p.dx
    b = Bunch(nb_tot=max(nb, 1), charge_pc=200.0, sxb=5.0, syb=3.0, gam=1957.0, epsy=1.0, epsz=1.0, dg=1.0,
              xc=p.xmn + 0.6 * lx, seed=77)
    rec = bunch_records(p, b, n0_ref=0.1) if nb > 0 else None
    dev = PicDevice(p)
    dev.env_enable(env_params(g, 0.8, 2))
    dev.set_plasma_source(plasma(0, 2, 2, 1, -1, 0.25, x_start=p.gxmin, x_end=1.0e7, y_min=p.gymin, y_max=p.gymax,
                                 z_min=p.gzmin, z_max=p.gzmax, jitter=0.5, seed=20241206))
    dev.load_plasma(0)
    if rec is not None:
        rc = dev.beam_inject(0, rec, b.gam)
        if rc != 0:
            raise RuntimeError(f"agpu_beam_inject returned {rc}")
    n = dev.count(0)
    it = 0
    for _ in range(warmup):
        it += 1
        dev.env_run(it * p.dt, it)
    dev.set_profiling(True)
    dev.reset_timers()
    s = torch.cuda.ExternalStream(dev.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev.synchronize()
    e0.record(s)
    pushes = 0
    for _ in range(steps):
        it += 1
        o = dev.env_run(it * p.dt, it)
        pushes += o.np[0] + o.removed[0] - o.injected[0]
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    tm = dev.timers()
    dev.close()
    return {"grid": [nx, ny, nz], "bunch_macroparticles": nb, "particles": int(n), "form": "fp64",
            "route": "agpu_env_run (env_lpf2_evolve + window), envelope solver on a zero envelope",
            "pushes_per_s": pushes / (ms * 1e-3), "ms_per_step": ms / steps,
            "particle_kernels_ms_per_step": tm.ms_push_deposit / steps, "yee_ms_per_step": tm.ms_yee / steps,
            "warmup": warmup, "steps": steps, "error_bits": int(o.error_bits)}


def tune_scan(torch, n_tune=32, warmup=3, steps=5):
    """The batch's worker threads and sort interval chosen by the tuner
    (aladyn_b200/autotune.py) on the first n_tune instances of the scan."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT
    from aladyn_b200.autotune import Tuner, tune_batch
    from aladyn_b200.sim import PicBatch
    cases = scan_instances(n_tune, AGPU_FP32_SPLIT)
    for p, _, _ in cases:
        p.capacity[0] = int(p.capacity[0] * 1.5)

    def make():
        b = PicBatch([c[0] for c in cases])
        for d, (p, las, src) in zip(b.instances, cases):
            d.init_laser(las)
            d.set_plasma_source(src)
            d.load_plasma(0)
        return b

    return tune_batch(torch, make, cases[0][0], 4, n_tune, warmup, steps, tuner=Tuner(None))


def extra_scan(torch, warmup, steps):
    tuned = tune_scan(torch)
    r = scan_measure(torch, warmup, steps, int(tuned.best["threads"]), sort_interval=int(tuned.best["sort_interval"]))
    return {"instances": r["n"], "warmup": warmup, "steps": steps,
            "batched_instance_steps_per_s": r["value"], "sequential_instance_steps_per_s": r["sequential"],
            "batched_over_sequential": r["value"] / r["sequential"],
            "sequential_path": "agpu_step per instance, one after the other, deferred counts and step graphs",
            "batched_options": tuned.best,
            "tuning": dict(tuned.as_dict(), note="worker threads and sort interval measured on the first "
                           "32 instances (5 steps each), the fastest applied to the 256-instance batch"),
            "batched_gpu_launches": int(r["launches_b"])}


def extra_continuity(torch):
    """Discrete continuity residual of one step (rho1 - rho0 + c div J_raw,
    FP64 on the host from the records before and after the step and the
    step's currents) relative to max |rho|, both forms, on the 3D
    128x64x64 and the 2D 1024x256 workloads, step 8 (the laser is in the
    plasma, no window shift yet); nodes within 5 of the array edges (folded
    ghost currents, box-edge removal) are left out."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
    from aladyn_b200.conservation import step_residual
    out = {"definition": "max|rho1 - rho0 + c div J_raw| / max|rho0|, c = 1/3 (3D), 1/2 (2D), one step"}
    for name in ("lwfa3d_128x64x64_ppc8", "lwfa2d_1024x256_ppc4"):
        res = {}
        for key, prec in (("fp32_split", AGPU_FP32_SPLIT), ("fp64", AGPU_FP64)):
            dev, p, las, src, ppc = load_device(name, prec)
            t = 0.0
            for it in range(8):  # the first window shift comes at step 10
                dev.lp_run(t, it, initial_time=(it == 0))
                t += p.dt
            part0 = dev.get_species(0)
            dev.lp_run(t, 8)
            part1 = dev.get_species(0)
            q = type(p).from_buffer_copy(p)
            q.xmn = dev.window_state()[3]
            r, rho, divj = step_residual(q, part0, part1, dev.get_currents(), margin=5)
            res[key] = {"residual_rel": r / rho, "max_c_div_j_rel": divj / rho}
            dev.close()
        out[name] = res
    return out


def extra_accuracy(torch, steps=1000):
    """FP32 split vs FP64 field error after a long run on the physical box of
    the 1024x256x256 workload at 3/8 of its resolution (384x96x96 cells, 8
    ppc, 2.8e7 electrons, moving window): relative L2 per component."""
    from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
    name = "lwfa3d_384x96x96_ppc8"
    f = {}
    for key, prec in (("fp64", AGPU_FP64), ("fp32_split", AGPU_FP32_SPLIT), ("fp64_rerun", AGPU_FP64)):
        dev, p, las, src, ppc = load_device(name, prec, cap_factor=1.6)
        t = 0.0
        for it in range(steps):
            dev.lp_run(t, it, initial_time=(it == 0))
            t += p.dt
        f[key] = (dev.get_fields(), dev.count(0))
        dev.close()

    def total(fa, fb):
        sl = (slice(2, p.nx + 2), slice(2, p.ny + 2), slice(2, p.nz + 2), slice(None))
        return float(np.linalg.norm(fa[sl] - fb[sl]) / np.linalg.norm(fb[sl]))

    err = rel_l2_errors(f["fp32_split"][0], f["fp64"][0], p)
    ctl = rel_l2_errors(f["fp64_rerun"][0], f["fp64"][0], p)
    return {"workload": name, "steps": steps, "rel_l2_per_component": err, "max": max(err),
            "rel_l2_all_components": total(f["fp32_split"][0], f["fp64"][0]),
            "fp64_rerun_rel_l2_per_component": ctl,
            "fp64_rerun_rel_l2_all_components": total(f["fp64_rerun"][0], f["fp64"][0]),
            "control_note": "a second FP64 run differs from the first only by the order of its atomic sums",
            "electrons": {k: int(v[1]) for k, v in f.items()}}


def extras(torch, warmup, only=None):
    k = 5
    todo = {
        "c1_2d": (extra_c1, torch, warmup, 20),
        "c2_cubic": (extra_forms, "lwfa3d_1024x256x256_ppc8_cubic", torch, warmup, k),
        "c3_pwfa": (extra_pwfa, torch, warmup, k),
        "c3_pwfa_envelope": (extra_pwfa_envelope, torch, warmup, k),
        "c4_ionization": (extra_ionization, torch, warmup, k),
        "scan": (extra_scan, torch, warmup, 10),
        "continuity_residual": (extra_continuity, torch),
        "accuracy_1000_steps": (extra_accuracy, torch),
    }
    # small cases for profiler captures, run only when named
    captures = {
        "pwfa_envelope_192x96x96_plasma": (extra_pwfa_envelope, torch, warmup, 3, 192, 96, 96, 0),
    }
    if only in captures:
        return {only: _guard(*captures[only])}
    return {name: _guard(*job) for name, job in todo.items() if only is None or name == only}


def bench_scan(a, torch):
    clk = ClockSampler(torch.cuda.current_device())
    if not a.no_clocks:
        clk.start()
    r = scan_measure(torch, a.warmup, a.steps, a.scan_threads)
    clocks = clk.stop()
    n = r["n"]
    line = {"metric": "instance-steps/s", "value": r["value"], "unit": "instance-steps/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": r["ms_b"] / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-split",
            "data": "synthetic: seeded instance draws, jittered lattice plasma, Gaussian lasers",
            "config": {"workload": SCAN_WORKLOAD, "instances": n, "nx": list(SCAN_NX), "ny": list(SCAN_NY),
                       "ppc": 4, "cells_total": r["cells"], "window": "moving, w_sh=10",
                       "threads": a.scan_threads or os.cpu_count()},
            "sequential": {"value": r["sequential"], "unit": "instance-steps/s", "ms_per_step": r["ms_s"] / a.steps,
                           "path": "agpu_step per instance, one instance after the other, deferred counts and "
                                   "step graphs"},
            "batched_over_sequential": r["value"] / r["sequential"],
            "pushes_per_s": {"batched": r["pushes_b"] / (r["ms_b"] * 1e-3),
                             "sequential": r["pushes_s"] / (r["ms_s"] * 1e-3)},
            "gpu_launches": int(r["launches_b"]), "clocks": clocks}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS) + [SCAN_WORKLOAD])
    ap.add_argument("--scan-threads", type=int, default=0, help="batch worker threads (0 = host cores)")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-clocks", action="store_true", help="skip nvidia-smi sampling (profiler runs)")
    ap.add_argument("--no-extras", action="store_true", help="only the headline workload")
    ap.add_argument("--extra", default=None, help="run one of the extra measurements alone and print it")
    a = ap.parse_args(argv)
    a.warmup = max(a.warmup, 3)
    if a.extra:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({a.extra: extras(torch, a.warmup, only=a.extra)[a.extra]}), flush=True)
        return 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.workload == SCAN_WORKLOAD:
        if a.impl == "reference" or world > 1:
            if rank == 0:
                print(json.dumps({"impl": a.impl, "workload": SCAN_WORKLOAD,
                                  "unavailable": "the scan is measured as batched vs sequential on one GPU"}))
            return 0
        import torch
        torch.cuda.set_device(local)
        return bench_scan(a, torch)
    w = WORKLOADS[a.workload]
    ppc_w = w["ppc"][0] * w["ppc"][1] * (w["ppc"][2] if w["ndim"] == 3 else 1)
    shapes = ("cubic on integer nodes, quadratic on half nodes, cubic Esirkepov (extension)" if w.get("shape", 0)
              else "quadratic/linear staggered (reference qlh + Esirkepov)")
    config = {"workload": a.workload, "grid": [w["nx"], w["ny"], w["nz"]], "ppc": ppc_w,
              "shapes": shapes, "window": "moving, w_sh=10",
              "l2": "inputs larger than L2 (particle arrays of tens of GB)", "replicas": world}
    metric = "particle-pushes/s"

    if a.impl == "reference":
        if rank != 0:
            return 0
        r = cpu_sample(a.workload, warmup=a.warmup, steps=a.steps)
        line = {"metric": metric, "value": r["value"], "unit": "pushes/s", "n_gpus": a.gpus,
                "steps": r["steps"], "warmup": a.warmup, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": {"value": r["value"], "unit": "pushes/s", "cores": r["cores"], "kind": "port",
                                 "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": "pushes/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    barrier, maxred, sumred = make_reducers(torch, world, "cuda")

    from aladyn_b200.abi import AGPU_FP32_SPLIT, AGPU_FP64
    clk = ClockSampler(torch.cuda.current_device() if world == 1 else local)
    if not a.no_clocks:
        clk.start()
    r32 = run_form(a.workload, AGPU_FP32_SPLIT, a.warmup, a.steps, torch, barrier, keep_fields=(world == 1))
    r64 = run_form(a.workload, AGPU_FP64, a.warmup, a.steps, torch, barrier, keep_fields=(world == 1))
    clocks = clk.stop()
    err = None
    if r32["fields"] is not None and r64["fields"] is not None:
        err = rel_l2_errors(r32["fields"], r64["fields"], r32["p"])
        r32["fields"] = r64["fields"] = None
    ms32 = maxred(r32["ms"])
    ms64 = maxred(r64["ms"])
    pushes32 = sumred(r32["pushes"])
    pushes64 = sumred(r64["pushes"])
    value = pushes32 / (ms32 * 1e-3)
    value64 = pushes64 / (ms64 * 1e-3)

    e2e = None
    if not a.no_e2e:
        r = run_e2e(a.workload, AGPU_FP32_SPLIT, a.warmup, a.steps, torch, barrier)
        ms = maxred(r["ms"])
        e2e = {"value": sumred(r["pushes"]) / (ms * 1e-3), "unit": "pushes/s",
               "h2d_bytes_per_step": int(r["h2d"]), "d2h_bytes_per_step": int(r["d2h"]),
               "path": "agpu_step + agpu_window_inject (pinned host records) + agpu_diag per step"}

    peak, peak_kind = measured_peaks()
    tm = r32["timers"]
    bpp = bytes_per_push(w["ndim"], ppc_w, True)
    ms_push = tm.ms_push_deposit
    achieved = bpp * tm.pushes / (ms_push * 1e-3) / 1e9 if ms_push > 0 else None
    p = r32["p"]
    cells = p.nx * p.ny * (p.nz if p.ndim == 3 else 1)
    yee32 = yee_bytes_per_cell(p.ndim, True) * cells * a.steps / (tm.ms_yee * 1e-3) / 1e9 if tm.ms_yee else None
    tm64 = r64["timers"]
    yee64 = yee_bytes_per_cell(p.ndim, False) * cells * a.steps / (tm64.ms_yee * 1e-3) / 1e9 if tm64.ms_yee else None
    push64 = bytes_per_push(w["ndim"], ppc_w, False) * tm64.pushes / (tm64.ms_push_deposit * 1e-3) / 1e9

    more = {}
    if world == 1 and not a.no_extras and a.workload == DEFAULT_WORKLOAD:
        more = extras(torch, a.warmup)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        c = cpu_sample(a.workload, budget_s=a.cpu_budget)
        cpu = {"value": c["value"], "unit": "pushes/s", "cores": c["cores"], "kind": "port", "sample": c["sample"]}

    if rank == 0:
        line = {
            "metric": metric, "value": value, "unit": "pushes/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms32 / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-split (int node + f32 offset, f32 fields/momenta/currents)",
            "data": "synthetic: seeded jittered lattice plasma + Gaussian laser", "config": config,
            "fp64": {"value": value64, "unit": "pushes/s", "ms_per_step": ms64 / a.steps,
                     "push_deposit_gbs": push64, "yee_gbs": yee64},
            "fp32_over_fp64": value / value64,
            "field_error_fp32_vs_fp64": {"rel_l2_per_component": err, "after_steps": a.warmup + a.steps},
            "yee_gbs": {"fp32": yee32, "fp64": yee64,
                        "note": "algorithmic 15 words/cell over the Yee phase (boundaries, current fold, 3 sweeps)"},
            "roofline": {"bound": "hbm", "kernel": "k32_tile (gather+push+deposit, FP32 split)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                         "bytes_per_push": bpp,
                         "traffic": (K32_DRAM_BYTES_PER_PUSH * tm.pushes / max(1, tm.launches_push_deposit)
                                     if w["ndim"] == 3 and ppc_w == 8 and not w.get("shape", 0) else None),
                         "traffic_note": "ncu dram bytes per particle of a small capture, scaled to the launch"},
            "phase_ms_per_step": {"push_deposit": tm.ms_push_deposit / a.steps, "yee": tm.ms_yee / a.steps,
                                  "sort_compact": tm.ms_sort / a.steps, "window": tm.ms_window / a.steps},
            "gpu_launches": int(tm.launches_total),
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "error_bits": r32["err"] | r64["err"],
        }
        line.update(more)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
