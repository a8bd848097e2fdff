"""Benchmark of the per-patch explicit FV step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

Workload (one periodic Cartesian patch of n^3 cells per GPU, default 256^3 =
16.8 M cells): uniform Mach 0.3 flow with an isentropic vortex (strength 5,
radius 0.1) and a Gaussian density pulse (1e-2, width 0.05); AUSM+ flux with
Upwind2 / van Albada reconstruction; 3-stage low-storage RK (alpha 1/4, 1/2,
1) at CFL 0.5.  A step is one RK time step (three stage launches).

Metric: Mcell-updates/s per RK stage = cells * 3 * K / time / 1e6, for the
FP32 bulk path (`value`) and the plain FP64 path (`fp64_plain`), with the
FP32 error against the FP64 run after the same steps and the FP32
conservation drift.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-updates/s per RK stage, FP32-batched vs FP64 plain at stated L2 error"
UNIT = "Mcell-updates/s"
STAGES = 3


def workload_name(n):
    return (f"single periodic patch {n}^3, Mach 0.3 flow + isentropic vortex (beta 5, R 0.1) + Gaussian "
            f"density pulse (1e-2, w 0.05), AUSM+ / Upwind2-VanAlbada / RK3 (1/4, 1/2, 1), CFL 0.5")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Polling loop of the clock sampler, run as its own process (its own
# interpreter lock: the timing thread may hold the parent's while it waits
# on the GPU).  argv: GPU UUID, output path.  NVML read-only queries only.
_CLOCK_POLLER = r"""
import sys, time, pynvml
pynvml.nvmlInit()
want = sys.argv[1].lower().replace("gpu-", "")
h = None
for q in range(pynvml.nvmlDeviceGetCount()):
    c = pynvml.nvmlDeviceGetHandleByIndex(q)
    u = pynvml.nvmlDeviceGetUUID(c)
    u = (u.decode() if isinstance(u, bytes) else u).lower().replace("gpu-", "")
    if u == want:
        h = c
if h is None:
    sys.exit(3)
smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
with open(sys.argv[2], "w", buffering=1) as f:
    f.write("time,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons\n")
    while True:
        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        pw = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
        f.write(f"{time.time():.6f},{sm},{smax},{pw:.1f},{rs}\n")
        time.sleep(0.001)
"""


class ClockSampler:
    """Samples the SM clock, power and clock-event reasons of this rank's GPU
    during a timed region: a separate process polls NVML's read-only queries
    about every millisecond, and the samples whose timestamps fall between
    start() returning and stop() being called are kept (the CSV file
    clocks_bench_rank<r>.csv in the --clock-dir directory holds them all).
    Falls back to nvidia-smi where NVML is unavailable."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvmlClocksEventReason*)
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device_index, out_dir):
        self.device_index = device_index
        self.proc = None
        self.mode = None
        self.path = os.path.join(out_dir, f"clocks_bench_rank{device_index}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device_index).uuid)
            if os.path.exists(self.path):
                os.remove(self.path)
            self.proc = subprocess.Popen([sys.executable, "-c", _CLOCK_POLLER, uuid, self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            # ready once the first sample is written (at most a few seconds)
            t_end = time.time() + 20.0
            while time.time() < t_end and self.proc.poll() is None:
                if os.path.exists(self.path) and sum(1 for _ in open(self.path)) >= 2:
                    self.mode = "nvml"
                    self.t0 = time.time()
                    return
                time.sleep(0.01)
            self._kill()
        except Exception:
            self._kill()
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            self.mode = "nvidia-smi"
        except OSError:
            self.proc = None

    def _kill(self):
        if self.proc is not None and self.proc.poll() is None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.proc = None

    def stop(self):
        if self.mode == "nvml":
            t1 = time.time()
            time.sleep(0.005)
            self._kill()
            sm, smax, reasons = [], [], set()
            for line in open(self.path).readlines()[1:]:
                parts = line.strip().split(",")
                if len(parts) < 5:
                    continue
                try:
                    t, c, cm, rs = float(parts[0]), float(parts[1]), float(parts[2]), int(parts[4])
                except ValueError:
                    continue
                if self.t0 <= t <= t1:
                    sm.append(c)
                    smax.append(cm)
                    reasons.update(nm for nm, bit in self.REASONS if rs & bit)
            if not sm:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                    "samples": len(sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self._kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


def _ref_rate(pyoracle, U0, h, dt, threads, precision, budget_s):
    """Reference RK steps on the host cores for about budget_s seconds:
    (Mcell-updates/s credited for the cells it computes, steps, computed
    cells).  The periodic harness adds two ghost layers per side, which the
    reference's iterator computes like interior cells, so they are credited."""
    s = pyoracle.RefSession(U0, h, threads=threads, precision=precision)
    sec = s.step(1, dt)
    steps = 1
    extra = int(max(0, min(3, budget_s / max(sec, 1e-3) - 1)))
    if extra:
        sec += s.step(extra, dt)
        steps += extra
    cells = s.computed_cells
    s.close()
    return cells * STAGES * steps / sec / 1e6, steps, cells


def cpu_baseline(U0, h, dt, budget_s=12.0):
    """The reference CPU iterator (compiled from its own sources) on the host
    cores, on a bounded sample of the same workload: in the reference's
    shipped single precision (`real` = float, drnum.h:43; the like-for-like
    baseline of the FP32-bulk path) and in FP64 (the build the parity tests
    pin)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    n = U0.shape[1]
    if pyoracle.ref_available() and pyoracle.ref_f32_available():
        threads = os.cpu_count() or 1
        out = {}
        for prec in ("f32", "f64"):
            v, steps, cells = _ref_rate(pyoracle, U0, h, dt, threads, prec, budget_s)
            out[prec] = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "precision": prec,
                         "sample": f"{steps} RK step(s) of the same {n}^3 periodic patch ({cells} cells computed with "
                                   f"the two ghost layers per side, credited), reference CartesianIterator + "
                                   f"RungeKutta compiled {'FP32 (as shipped)' if prec == 'f32' else 'FP64'}, "
                                   f"OpenMP {threads} threads, RungeKutta::operator() timed"}
        line = dict(out["f32"])
        line["fp64"] = out["f64"]
        return line
    # the restatement (single thread) on a smaller sample of the same physics
    from drnum_b200 import cases
    m = 64
    U, hh, dts = cases.periodic_box(m)
    t0 = time.perf_counter()
    pyoracle.oracle_run(U, hh, dts, 2)
    sec = time.perf_counter() - t0
    return {"value": m ** 3 * STAGES * 2 / sec / 1e6, "unit": UNIT, "cores": 1, "kind": "port", "precision": "f64",
            "sample": f"2 RK steps of a {m}^3 box of the same physics, oracle restatement (1 thread)"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (compiled reference
    library in its shipped single precision, all host threads), same config
    and metric as our arm; the FP64 build timed beside it."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from drnum_b200 import cases
    if not (pyoracle.ref_available() and pyoracle.ref_f32_available()):
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference library oracle/_ref is missing"}))
        return 0
    n = args.n
    U0, h, dt = cases.periodic_box(n)
    threads = os.cpu_count() or 1
    s = pyoracle.RefSession(U0, h, threads=threads, precision="f32")
    sample_n = n
    # calibrate with the first warm-up step; shrink the per-step sample if the
    # whole run would exceed about three minutes
    t_first = s.step(1, dt)
    if (args.warmup + args.steps) * t_first > 180.0 and n > 128:
        s.close()
        sample_n = 128
        U0, h, dt = cases.periodic_box(sample_n)
        s = pyoracle.RefSession(U0, h, threads=threads, precision="f32")
        s.step(1, dt)
    for _ in range(max(0, args.warmup - 1)):
        s.step(1, dt)
    sec = s.step(args.steps, dt)
    cells = s.computed_cells
    value = cells * STAGES * args.steps / sec / 1e6
    s.close()
    v64, steps64, _ = _ref_rate(pyoracle, U0, h, dt, threads, "f64", 10.0)
    sample = (f"each step one RK step (3 stages) of a periodic {sample_n}^3 patch of the workload "
              f"({cells} cells computed with the two ghost layers per side, credited), reference CartesianIterator + "
              f"RungeKutta compiled from its own sources in its shipped single precision, OpenMP {threads} threads")
    config = {"workload": workload_name(sample_n), "cells": sample_n ** 3, "cells_computed": cells}
    if sample_n != n:
        config["note"] = f"sample reduced from {n}^3 to {sample_n}^3 to bound the run time"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "precision": "f32", "sample": sample,
                             "fp64": {"value": v64, "unit": UNIT, "steps": steps64,
                                      "sample": "the FP64 build of the same code on the same patch"}},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from drnum_b200 import _lib, cases
    from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.n
    U0, h, dt = cases.periodic_box(n)
    cells = n ** 3
    # a dedicated (non-default) stream: the library's kernels and the timing
    # events are issued on it
    stream = torch.cuda.Stream(dev)

    def make(precision):
        patch = CartesianPatch(n, n, n, spacing=(h, h, h))
        patch.setField(0, U0)
        it = B200CartesianIterator(AusmPlus(), local_rank, precision)
        it.addPatch(patch)
        it.updateDevice(fields=(0,))
        it.sync()
        _lib.check(it.ctx, it.lib.dn_set_stream(it.ctx, ctypes_void(stream.cuda_stream)))
        return patch, it

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_steps(it, k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize(dev)
        l0 = it.launchCount()
        e0.record(stream)
        for _ in range(k):
            it.rkStep(dt, cases.RK3_ALPHA)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        return e0.elapsed_time(e1) / 1e3, it.launchCount() - l0

    # ---- FP32 bulk (headline)
    p32, it32 = make(_lib.DN_FP32)
    # schedule autotune (plane-chunk length of the stage CTAs; changes no
    # result), before the warm-up and outside every timed region
    it32.autotune()
    s0 = it32.conservationSums()
    for _ in range(args.warmup):
        it32.rkStep(dt, cases.RK3_ALPHA)
    it32.sync()
    clocks = ClockSampler(local_rank, args.clock_dir)
    clocks.start()
    t32, launches = timed_steps(it32, args.steps)
    clock_info = clocks.stop()
    it32.sync()
    s1 = it32.conservationSums()
    t32 = max_over_ranks(t32)
    value = world * cells * STAGES * args.steps / t32 / 1e6

    # ---- plain FP64, same steps from the same initial state
    p64, it64 = make(_lib.DN_FP64)
    for _ in range(args.warmup):
        it64.rkStep(dt, cases.RK3_ALPHA)
    it64.sync()
    t64, _ = timed_steps(it64, args.steps)
    t64 = max_over_ranks(t64)
    value64 = world * cells * STAGES * args.steps / t64 / 1e6

    # ---- error of the FP32 run against the FP64 run after warmup + steps
    it32.updateHost(fields=(0,))
    it64.updateHost(fields=(0,))
    a, b = p32.getField(0), p64.getField(0)
    drho = (a[0] - b[0]) / cases.RHO_INF
    pa = cases.cons_to_prim(a)[0]
    pb = cases.cons_to_prim(b)[0]
    dp = (pa - pb) / cases.P_INF
    err = {"l2_rho_rel": float(np.sqrt(np.mean(drho ** 2))), "linf_rho_rel": float(np.abs(drho).max()),
           "l2_p_rel": float(np.sqrt(np.mean(dp ** 2))), "linf_p_rel": float(np.abs(dp).max()),
           "steps": args.warmup + args.steps, "against": "FP64 plain GPU path (bit-identical to the reference CPU iterator)"}
    drift = [float((s1[v] - s0[v]) / abs(s0[v])) if s0[v] != 0 else float(s1[v] - s0[v]) for v in range(5)]
    it64.close()
    del p64, a, b

    # ---- e2e through the C ABI with pinned host buffers (float, the reference's default `real`):
    # every step uploads its input state from the host and reads its result back; the
    # asynchronous calls let the read-back of step k, the upload of step k+1 and the
    # stages of step k+1 overlap (two copy engines, two staging buffers each way)
    hin = [torch.empty((5, n, n, n), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    hout = [torch.empty((5, n, n, n), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    for b in hin:
        b[...] = p32.getField(0).astype(np.float32)
    ctx, lib = it32.ctx, it32.lib
    fin = [_lib.fptr(b) for b in hin]
    fout = [_lib.fptr(b) for b in hout]
    alpha = np.ascontiguousarray(cases.RK3_ALPHA, dtype=np.float64)

    def e2e_step(k):
        _lib.check(ctx, lib.dn_patch_upload_f32_async(ctx, 0, 0, fin[k % 2]))
        _lib.check(ctx, lib.dn_rk_step(ctx, dt, _lib.dptr(alpha), 3))
        _lib.check(ctx, lib.dn_patch_download_f32_async(ctx, 0, 0, fout[k % 2]))

    for k in range(min(args.warmup, 3)):
        e2e_step(k)
    _lib.check(ctx, lib.dn_sync(ctx))
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        e2e_step(k)
    _lib.check(ctx, lib.dn_sync(ctx))      # all copies of the last step have landed
    e1.record(stream)
    torch.cuda.synchronize(dev)
    te = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e_value = world * cells * STAGES * args.steps / te / 1e6
    it32.close()

    # ---- roofline of the dominant kernel (the FP32 stage kernel)
    peak, peak_kind = measured_peaks()
    bytes_per_launch = 60.0 * cells      # read f(k-1) + read f(n) + write f(k), 5 x FP32 each
    launch_s = t32 / (STAGES * args.steps)
    achieved = bytes_per_launch / launch_s / 1e9
    # DRAM traffic of the kernel per launch, from one ncu capture of the three
    # stage launches of a timed RK step on the periodic 192^3 patch
    # (dram__bytes_read + dram__bytes_write: 36.6, 58.1 and 58.2 B per cell;
    # stage 1 reads f(k-1) = f(n) once), averaged and scaled by the cells of
    # this launch: the kernel streams each plane once, so the traffic grows
    # with the cell count
    TRAFFIC_BYTES_PER_CELL = 50.9
    traffic = TRAFFIC_BYTES_PER_CELL * cells

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(U0, h, dt)

    # ---- the multi-patch workloads (overlap interpolation, boundary fluxes,
    # level-set wall, many uneven patches): on one GPU each workload whole;
    # on several GPUs each workload sharded over the ranks (its patches
    # partitioned, compact shadows, NCCL exchange of donor cells) and the
    # periodic patch split into one i-slab per rank
    extra, sharded = {}, {}
    names = [w for w in args.workloads.split(",") if w]
    if world == 1 and not args.sharded:
        for name in names:
            extra[name] = run_workload(name, args, dev, stream, rank, world, barrier, max_over_ranks)
    else:
        for name in (["slab"] if world > 1 else []) + names:
            sharded[name] = run_sharded(name, args, dev, rank, world, barrier, max_over_ranks)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t32 / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (int32 fixed-point storage)", "data": "synthetic",
            "config": {"workload": workload_name(n), "cells_per_gpu": cells, "stages_per_step": STAGES,
                       "dt": dt, "l2": "inputs larger than L2 (each field 5 x 4 B x cells = "
                                         f"{20 * cells / 1e6:.0f} MB per GPU)",
                       "parallelism": f"one independent patch per GPU (x{world}), no collective on the data path",
                       "tuning": "dn_autotune before the warm-up: plane-chunk length of the stage CTAs"},
            "fp64_plain": {"value": value64, "unit": UNIT, "ms_per_step": t64 / args.steps * 1e3,
                           "fp32_over_fp64": value / value64},
            "error_vs_fp64": err,
            "conservation_drift_rel": {"mass": drift[0], "mom_x": drift[1], "mom_y": drift[2], "mom_z": drift[3],
                                       "energy": drift[4], "steps": args.warmup + args.steps},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "fx_stage_kernel<16,32> (FP32 arithmetic in packed f32x2 pairs, int32 fixed-point storage)",
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": launch_s * 1e3},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 20 * cells,
                    "d2h_bytes_per_step": 20 * cells,
                    "path": "dn_patch_upload_f32_async (pinned host) + dn_rk_step + dn_patch_download_f32_async per step, dn_sync at the end"},
            "gpu_launches": int(launches),
            "clocks": clock_info,
            "workloads": extra,
        }
        if sharded:
            line["sharded"] = sharded
        print(json.dumps(line), flush=True)
    return 0


def run_workload(name, args, dev, stream, rank, world, barrier, max_over_ranks):
    """One multi-patch workload (drnum_b200.workloads): FP32 bulk batched
    (autotuned tiles, CUDA-graph steps) and plain FP64 from the same state,
    timed over args.steps steps after args.warmup; error of FP32 against FP64."""
    import torch
    from drnum_b200 import _lib, cases, workloads

    case = workloads.build(name, args.workload_scale)
    grid, objs = workloads.make_grid(case)
    del case["states"]
    cells = sum(int(np.prod(p["n"])) for p in case["patches"])
    out = {"description": case["description"], "patches": len(case["patches"]), "cells": cells,
           "no_donor_cells": grid.no_donor, "steps": args.steps, "warmup": args.warmup, "dt": case["dt"]}
    its = {}
    for prec in (_lib.DN_FP32, _lib.DN_FP64):
        it = workloads.make_iterator(objs, prec, dev.index)
        _lib.check(it.ctx, it.lib.dn_set_stream(it.ctx, ctypes_void(stream.cuda_stream)))
        it.setOption(_lib.DN_OPT_GRAPH, 1)
        its[prec] = it
    if case["levelset"] is not None:
        out["levelset_layer_cells"] = int(sum(len(layer["cells"]) for q in range(len(objs))
                                              for layer in its[_lib.DN_FP32].levelSetLayers(q)["inner"]))
    out["tile_costs_ns_per_padded_cell"] = [float(x) for x in its[_lib.DN_FP32].autotune()]
    dt = case["dt"]
    res = {}
    for prec, key in ((_lib.DN_FP32, "fp32_batched"), (_lib.DN_FP64, "fp64_plain")):
        it = its[prec]
        for _ in range(args.warmup):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize(dev)
        l0 = it.launchCount()
        e0.record(stream)
        for _ in range(args.steps):
            it.rkStep(dt, cases.RK3_ALPHA)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        it.sync()
        mcell = world * cells * STAGES * args.steps / t / 1e6
        bpc = 60.0 if prec == _lib.DN_FP32 else 120.0
        res[key] = {"value": mcell, "unit": UNIT, "ms_per_step": t / args.steps * 1e3,
                    "launches_per_step": (it.launchCount() - l0) / args.steps,
                    "algorithmic_gbs": mcell * 1e6 * bpc / 1e9}
        if case["levelset"] is not None:
            # FP64 residual norm of the last step, Patch::computeVariableDifference
            # of density between field 0 and the step-start field 1
            mx, l2 = 0.0, 0.0
            for q in range(len(objs)):
                a, b = it.computeVariableDifference(q, 0, 0, 1, 0)
                mx, l2 = max(mx, a), l2 + b * b
            res[key]["residual_norms_rho"] = {"max": mx, "l2": float(np.sqrt(l2))}
    peak, _ = measured_peaks()
    res["fp32_batched"]["hbm_frac_of_measured"] = res["fp32_batched"]["algorithmic_gbs"] / peak
    out.update(res)
    out["fp32_over_fp64"] = res["fp32_batched"]["value"] / res["fp64_plain"]["value"]
    # error of the FP32 run against the FP64 run after warmup + steps
    num_r = num_p = den = 0.0
    lin_r, lin_p = [], []
    nonfinite = 0
    for q in range(len(objs)):
        a = its[_lib.DN_FP32].downloadField(q, 0)
        b = its[_lib.DN_FP64].downloadField(q, 0)
        nonfinite += int((~np.isfinite(a)).sum() + (~np.isfinite(b)).sum())
        dr = (a[0] - b[0]) / cases.RHO_INF
        dp = (cases.cons_to_prim(a)[0] - cases.cons_to_prim(b)[0]) / cases.P_INF
        num_r += float((dr ** 2).sum())
        num_p += float((dp ** 2).sum())
        den += dr.size
        lin_r.append(float(np.abs(dr).max()))
        lin_p.append(float(np.abs(dp).max()))
    out["error_vs_fp64"] = {"l2_rho_rel": float(np.sqrt(num_r / den)), "linf_rho_rel": float(np.max(lin_r)),
                            "l2_p_rel": float(np.sqrt(num_p / den)), "linf_p_rel": float(np.max(lin_p)),
                            "nonfinite_values": nonfinite, "steps": args.warmup + args.steps}
    for it in its.values():
        it.close()
    return out


def run_sharded(name, args, dev, rank, world, barrier, max_over_ranks):
    """One workload sharded over the ranks (strong scaling: the whole grid's
    cells are fixed): patches partitioned by cell count (`slab`: the periodic
    n^3 patch split into one i-slab per rank), each rank holding its own
    patches and compact shadows of the donor cells it reads, donor cells
    exchanged by NCCL send/recv before every donor copy (drnum_b200.shard).
    FP32 bulk; timed over args.steps steps after args.warmup, max over ranks."""
    import torch
    from drnum_b200 import _lib, cases, shard, workloads
    tables = None
    if name == "slab":
        U0, h, dt = cases.periodic_box(args.n)
        slabs = shard.slab_split((args.n,) * 3, world)
        objs = shard.slab_patches(U0, h, slabs)
        tables = [s["tables"] for s in slabs]
        owner = list(range(world))
        cells = args.n ** 3
        desc = (f"periodic {args.n}^3 patch of the headline workload split into {world} i-slabs (2 seek planes "
                "per side, copied from the neighbouring slab before every stage)")
    else:
        case = workloads.build(name, args.workload_scale)
        _, objs = workloads.make_grid(case)
        dt = case["dt"]
        cells = sum(int(np.prod(p["n"])) for p in case["patches"])
        owner = shard.partition([int(np.prod(p["n"])) for p in case["patches"]], world)
        desc = case["description"]
        del case
    # one dn_rk_step per step (the level-set wall of the sphere is the
    # context's own post-operation), the exchange in its donor-copy hook
    sh = shard.make_sharded(objs, owner, rank, world, _lib.DN_FP32, dev.index, compact=True, tables=tables)
    if any(o == rank for o in owner):
        sh.it.autotune()
    for _ in range(args.warmup):
        sh.rkStep(dt, cases.RK3_ALPHA)
    torch.cuda.synchronize(dev)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(sh.stream)
    for _ in range(args.steps):
        sh.rkStep(dt, cases.RK3_ALPHA)
    e1.record(sh.stream)
    torch.cuda.synchronize(dev)
    barrier()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    held = max_over_ranks(float(sh.deviceCells()))
    exchanges = 2 * len(cases.RK3_ALPHA)        # one before every donor copy of dn_rk_step
    sent = max_over_ranks(float(sum(n_send for n_send, _ in sh.counts.values()) * 5 * 4 * exchanges))
    sums = sh.conservationSums()
    sh.close()
    sh.it.close()
    value = cells * STAGES * args.steps / t / 1e6
    return {"description": desc, "cells": cells, "patches": len(objs), "ranks": world, "scaling": "strong",
            "value": value, "unit": UNIT, "ms_per_step": t / args.steps * 1e3, "steps": args.steps,
            "warmup": args.warmup, "max_device_cells_per_rank": held,
            "device_cells_fraction_of_grid": held / cells,
            "exchange_bytes_per_step_max_rank": sent, "mass_sum": float(sums[0])}


def ctypes_void(x):
    import ctypes
    return ctypes.c_void_p(x)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clock-dir", default=os.environ.get("DN_CLOCK_DIR", tempfile.gettempdir()),
                    help="directory of the clock-sample CSV written during the timed region")
    ap.add_argument("--workloads", default="jet,sphere,tiled",
                    help="comma-separated multi-patch workloads to add to the line ('' for none)")
    ap.add_argument("--workload-scale", type=float, default=1.0,
                    help="linear scale of the multi-patch workloads (1 = the full-size cases)")
    ap.add_argument("--sharded", action="store_true",
                    help="run the multi-patch workloads through the sharded path also on one GPU "
                         "(always on several GPUs)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    group = world > 1 or args.sharded
    if group:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        kw = {}
        if world == 1:
            # a group of one for the sharded path on one GPU
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                port = sk.getsockname()[1]
            kw = {"init_method": f"tcp://127.0.0.1:{port}", "world_size": 1, "rank": 0}
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank), **kw)
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if group:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
