#!/usr/bin/env python
"""Throughput of the B200 FDTD time step on the 512^3 rough Drude-silver surface.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one "step" = one full Yee time step of the whole grid): 512^3 cells,
dx = 5 nm, dt = 0.5 x the 3D Courant limit, 16-cell CPML on all faces, a
Gaussian-correlated rough surface (rms 10 nm, correlation 50 nm, seed 2024)
with Drude silver (eps_inf 3.7, wp 1.38e16 rad/s, gamma 2.73e13 1/s) below and
vacuum above, a p-polarised TSF plane wave at 30 deg incidence (600 nm pulse),
three probes, and running DFTs at 500/600/700 nm on the NFFF box for a
91 x 181 far-field grid.  Inputs are synthetic (seeded height map), built by
gsvit_copy_b200.plan.rough_surface_scene.  Metric: Gcell-updates/s (cells x
steps / device time), higher is better.

Arms:
  --impl b200       the CUDA library through its C ABI (default).  Prints one
                    JSON line with value (device-timed steps, fields resident in
                    HBM, replayed from CUDA graphs by fdtd_step_graph), e2e (the
                    same job through the public Solver API with pinned host
                    buffers: initial fields uploaded, K steps, probes and final E
                    read back), the roofline of the dominant kernel, the clocks
                    seen and a CPU baseline.
  --impl reference  GSvit's own CPU stepping code (yee.c, boundary.c, source.c,
                    farfield.c ... compiled from its sources into
                    oracle/_ref/libgsvit_ref.so) on all host threads, on a
                    bounded sample of the same workload (see SAMPLE below).
                    The line also carries `reference_cuda`: GSvit's own CUDA
                    path (gpu.c + gpu_kernels.cu built unmodified for sm_100a,
                    oracle/_ref/libgsvit_refcuda.so) timed on this GPU, the
                    whole workload on a 256^3 sample and the field update at
                    the full size (context, not the arm's value).

Multi-GPU: the time step does not shard here; `--gpus N` under torchrun runs N
independent replicas (one per rank and GPU), timed as the max over ranks, and
`value` is the sum of all ranks' cell updates over that time (weak scaling).
The field arrays (3.2 GB per set) are far larger than L2, so no L2 flush is
needed between steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Gcell-updates/s"
# steps per CUDA graph of the timed runs (fdtd_step_graph); at 512^3 the
# replayed step is 2.70 ms against 2.75 ms launched eagerly
GRAPH_CHUNK = 32
UNIT = "Gcell/s"
# bounded CPU sample of the workload: same scene recipe at 128^3 with the far
# grid scaled with the edge length (46 x 91 points), so that the far-field
# work per cell update matches the 512^3 case
SAMPLE_RES = 128
SAMPLE_ANGLES = (46, 91)
SAMPLE_DESC = ("rough Drude-silver surface scene at 128^3 (dx 5 nm, 16-cell CPML, TSF 30 deg, "
               "NFFF 3 wavelengths on a 46x91 far grid: far work per cell update as at 512^3)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--res", type=int, default=512)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="reference arm: skip the context run of GSvit's own CUDA build")
    ap.add_argument("--refcuda-steps", type=int, default=5,
                    help="reference arm: timed steps of GSvit's own CUDA build with its far field")
    ap.add_argument("--no-extensions", action="store_true",
                    help="skip the extensions block (FP16 / BF16 storage and the batched instances)")
    ap.add_argument("--ext-steps", type=int, default=20, help="timed steps of each extensions measurement")
    ap.add_argument("--adj-steps", type=int, default=4000, help="adjoint workload: forward steps")
    ap.add_argument("--fd-cells", type=int, default=16, help="adjoint workload: cells checked by finite differences")
    ap.add_argument("--fd-h", type=float, default=1e-3, help="adjoint workload: finite-difference step on eps_r")
    ap.add_argument("--fd-storage", choices=["f64", "f32"], default="f64",
                    help="adjoint workload: field storage of the finite-difference runs")
    ap.add_argument("--prec-steps", type=int, default=4000, help="precision workload: steps of every run")
    ap.add_argument("--workload", choices=["rough512", "batched", "adjoint", "precision"], default="rough512",
                    help="batched: 48 uneven rough-surface instances in one batch against the same run one by one; "
                         "precision: FP32 / FP16 / BF16 storage against the FP64 reference-precision run")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class Replicas:
    """Plumbing of an N-rank run (torchrun, one process per GPU).  The ranks
    are independent replicas and exchange no data: a barrier on each side of
    the timed region and the slowest rank's time are all they share.  The GPU
    arm uses NCCL on its device; with one rank nothing is initialised."""

    def __init__(self, backend="nccl", device=None):
        import torch
        self.rank, self.local, self.world = dist_env()
        self.device = device if device is not None else torch.device("cpu")
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=300), **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        """The largest x over the ranks (every rank gets it)."""
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_gcells(cells_per_rank, steps, world, seconds):
    """Whole-job throughput: the cell updates of every rank over the slowest rank's time."""
    return cells_per_rank * steps * world / seconds / 1e9


def workload_scene(res, nsteps_planned):
    from gsvit_copy_b200 import plan
    return plan.rough_surface_scene(res=res, nsteps=nsteps_planned)


def sample_scene(nsteps_planned):
    from gsvit_copy_b200 import plan
    return plan.rough_surface_scene(res=SAMPLE_RES, nsteps=nsteps_planned, nfff_angles=SAMPLE_ANGLES)


def config_block(res, scene):
    return {
        "workload": f"rough Drude-silver surface {res}^3, 16-cell CPML, TSF 30 deg p-pol 600 nm, "
                    f"NFFF running DFT 3 wavelengths, 91x181 far grid, 3 probes",
        "cells": scene.ncells,
        "grid": [scene.xres, scene.yres, scene.zres],
        "planned_steps": scene.nsteps,
        "l2": "inputs larger than L2 (fields 3.2 GB per ping-pong set at 512^3); no flush",
        "timed_api": f"fdtd_step_graph (CUDA graphs of {GRAPH_CHUNK} steps, captured in the warm-up)",
        "parallelism": "replicas",
    }


# ----------------------------------------------------------------- clocks

CLOCK_FIELDS = ["index", "pci.bus_id", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
                "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
                "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while it runs (read only)."""

    def __init__(self, bus_id=None):
        self.bus_id = bus_id
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="clk", suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + ",".join(CLOCK_FIELDS), "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) != len(CLOCK_FIELDS):
                    continue
                if self.bus_id and self.bus_id.lower() not in p[1].lower() and p[1].lower() not in self.bus_id.lower():
                    continue
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[2]) for r in rows if num(r[2]) is not None]
        mx = [num(r[3]) for r in rows if num(r[3]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def bus_id_of(dev):
    import torch
    try:
        p = torch.cuda.get_device_properties(dev)
        dom, bus, d = getattr(p, "pci_domain_id", None), getattr(p, "pci_bus_id", None), getattr(p, "pci_device_id", None)
        if bus is not None:
            return "%08X:%02X:%02X" % (dom or 0, bus, d or 0)
    except Exception:
        pass
    return None


# ----------------------------------------------------------------- peaks / ncu figures

def hbm_peak():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(res, kernel="bulk_kernel"):
    """DRAM bytes per launch of `kernel` from the committed ncu summary of this workload."""
    path = os.path.join(HERE, "profiles", f"launches_rough{res}.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(f"{kernel} dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


KERNEL_NAMES = {
    "bulk": "tile_kernel, bulk layout (TMA-staged fused H+E step of the interior box)",
    "cpml": "tile_kernel, CPML layouts (TMA-staged fused H+E step with psi, kappa and ADE-in-CPML)",
}


def kernel_rooflines(prof, nprof, step_bytes, step_ms, peak, peak_kind, res):
    """Per-kernel figures of one step from fdtd_step_profile (CUDA events
    around each launch group): device ms, algorithmic bytes, achieved GB/s and
    the fraction of the HBM peak; the roofline block is the kernel with the
    largest share of the step."""
    total = prof["total_ms"] / nprof
    ks = {}
    for key, ms_key, b_key in (("bulk", "bulk_ms", "bulk_bytes"), ("cpml", "slab_ms", "slab_bytes")):
        ms = prof[ms_key] / nprof
        b = prof[b_key]
        gbs = b / (ms * 1e-3) / 1e9 if ms > 0 else None
        ks[key] = {"kernel": KERNEL_NAMES[key], "ms_per_launch": ms, "algorithmic_bytes": b, "achieved_gbs": gbs,
                   "frac": gbs / peak if gbs else None, "step_share": ms / total if total else None}
    ks["aux_tsf"] = {"kernel": "1D aux grid + TSF face tables", "ms_per_step": prof["aux_ms"] / nprof,
                     "step_share": prof["aux_ms"] / nprof / total if total else None}
    ks["nfff"] = {"kernel": "NFFF surface samples + running-DFT fold", "ms_per_step": prof["nfff_ms"] / nprof,
                  "step_share": prof["nfff_ms"] / nprof / total if total else None}
    top = max(("bulk", "cpml"), key=lambda k: ks[k]["ms_per_launch"])
    t = ks[top]
    roofline = {"kernel": t["kernel"], "bound": "hbm", "achieved": t["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": t["frac"], "peak_source": peak_kind,
                "traffic": ncu_traffic(res, "bulk_kernel" if top == "bulk" else "cpml_tiles"),
                "algorithmic_bytes": t["algorithmic_bytes"], "ms_per_launch": t["ms_per_launch"],
                "step_share": t["step_share"]}
    step_gbs = step_bytes / (step_ms * 1e-3) / 1e9
    return roofline, ks, {"achieved": step_gbs, "frac": step_gbs / peak, "bytes": step_bytes, "ms": step_ms}


# ----------------------------------------------------------------- CPU sample

def cpu_sample_run(steps=None, warmup=1, budget_s=15.0):
    """Time GSvit's own CPU stepping code (oracle/_ref) on the bounded sample.
    Returns (Gcell/s, threads, kind, steps timed)."""
    from oracle import pyoracle
    kind = "reference" if pyoracle.reference_available() else "port"
    scene = sample_scene(4000)
    cpu = pyoracle.CpuSolver(scene, "reference" if kind == "reference" else "oracle")
    cpu.step(warmup)
    if steps is None:
        t = time.perf_counter()
        cpu.step(1)
        one = time.perf_counter() - t
        steps = int(max(2, min(200, budget_s / max(one, 1e-6))))
    t = time.perf_counter()
    cpu.step(steps)
    dt = time.perf_counter() - t
    cpu.close()
    threads = int(os.environ.get("OMP_NUM_THREADS", 0)) or os.cpu_count()
    return scene.ncells * steps / dt / 1e9, threads, kind, steps


# GSvit's own CUDA path on this GPU (context, not the arm's value): the same
# scene recipe with the far grid scaled so that the far-field work per cell
# update is that of the 512^3 case (points proportional to the edge length)
REFCUDA_RES = 256
REFCUDA_ANGLES = (64, 129)


def reference_cuda_context(a):
    """Time GSvit's own CUDA build (src3d/gpu.c + gpu_kernels.cu compiled
    unmodified for sm_100a, oracle/_ref/libgsvit_refcuda.so) through the GPU
    branch of its loop, in a child process: the whole workload with its
    time-domain far field, and the field update alone (no NFFF).  Returns a
    block for the reference arm's line, or {"unavailable": why}."""
    from oracle import refcuda
    if not refcuda.available():
        return {"unavailable": "oracle/_ref/libgsvit_refcuda.so is not built (GSvit's sources absent at build time)"}
    if a.no_reference_cuda:
        return {"unavailable": "skipped (--no-reference-cuda)"}
    out = {"build": "GSvit src3d/gpu.c + src3d/gpu_kernels.cu, unmodified, nvcc -O2 -use_fast_math for sm_100a "
                    "(configure.ac:57), stepped through sv_pool_gpu_* (svit.c:240-256); FP32",
           "timing": "host clock around K steps; every reference stage ends in a device synchronisation"}
    try:
        full = refcuda.run("rough", REFCUDA_RES, steps=a.refcuda_steps, warmup=1, nfff=True, angles=REFCUDA_ANGLES,
                           timeout=900)
        bare = refcuda.run("rough", a.res, steps=2 * a.refcuda_steps, warmup=2, nfff=False, timeout=900)
    except Exception as e:   # the context block must not take the arm down
        return {"unavailable": f"reference CUDA run failed: {str(e)[-300:]}"}
    out["workload"] = {"value": full["gcells"], "unit": UNIT, "ms_per_step": full["ms_per_step"], "steps": full["steps"],
                       "sample": f"rough Drude-silver surface {REFCUDA_RES}^3, 16-cell CPML, TSF, time-domain NFFF on "
                                 f"{REFCUDA_ANGLES[0]}x{REFCUDA_ANGLES[1]} far points (far work per cell update as at 512^3)"}
    out["field_update"] = {"value": bare["gcells"], "unit": UNIT, "ms_per_step": bare["ms_per_step"],
                           "steps": bare["steps"], "sample": f"rough Drude-silver surface {a.res}^3 without the NFFF"}
    return out


def run_reference(a):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    refcuda_block = reference_cuda_context(a)
    value, threads, kind, steps = cpu_sample_run(steps=a.steps, warmup=a.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded height map)",
        "config": {"workload": f"rough Drude-silver surface {a.res}^3 (sampled: {SAMPLE_DESC})",
                   "sample_res": SAMPLE_RES},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{SAMPLE_DESC}, {steps} steps after {a.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["ms_per_step"] = SAMPLE_RES ** 3 / (value * 1e9) * 1e3
    line["reference_cuda"] = refcuda_block
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU arm

def run_b200(a):
    import torch
    from gsvit_copy_b200 import abi
    from gsvit_copy_b200.solver import Solver

    rank, local, world = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device (the library has no CPU path)")
    torch.cuda.set_device(local)
    ranks = Replicas("nccl", torch.device("cuda", local))
    barrier, max_over_ranks = ranks.barrier, ranks.max

    K, W = a.steps, a.warmup
    scene = workload_scene(a.res, max(4000, 2 * K + W + 160))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    g = Solver(scene, device=local)
    g.set_stream(stream.cuda_stream)

    # warm-up: W eager steps, then the CUDA graphs of GRAPH_CHUNK steps that
    # the timed runs replay (fdtd_step_graph), captured for both field-set
    # parities so that no capture falls inside a timed region
    g.step(W)
    for _ in range(2):
        g.step_graph(2 * GRAPH_CHUNK, chunk=GRAPH_CHUNK)
        g.step(1)
    g.sync()
    torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(bus_id_of(local)) as clk:
        e0.record(stream)
        g.step_graph(K, chunk=GRAPH_CHUNK)
        e1.record(stream)
        torch.cuda.synchronize()
    g.sync()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clocks = clk.summary()
    value = whole_job_gcells(scene.ncells, K, world, ms * 1e-3)

    # per-kernel profile of a few more steps (CUDA events around each launch)
    prof = g.step_profile(8)
    nprof = 8
    peak, peak_kind = hbm_peak()
    step_bytes = g.step_bytes()
    roofline, kernels, step_roof = kernel_rooflines(prof, nprof, step_bytes, ms / K, peak, peak_kind, a.res)
    # far-field integration of the accumulated running DFTs (once per run)
    t0 = time.perf_counter()
    spec = g.nfff_spectrum()
    ff_ms = (time.perf_counter() - t0) * 1e3
    # the step kernels of K steps, then the probe capture that closes fdtd_step
    gpu_launches = int(prof["launches_per_step"]) * K + (1 if scene.probes is not None and len(scene.probes) else 0)

    # end to end through the public API with pinned host buffers
    shape = g.shape
    host = [torch.empty(shape, dtype=torch.float32, pin_memory=True) for _ in range(6)]
    outE = [torch.empty(shape, dtype=torch.float32, pin_memory=True) for _ in range(3)]
    import ctypes as C
    ptrs = (C.POINTER(C.c_float) * 6)(*[C.cast(h.data_ptr(), C.POINTER(C.c_float)) for h in host])
    abi.check(g.lib.fdtd_get_fields_f32(g.h, abi.EH, ptrs), "fdtd_get_fields_f32")
    optrs = (C.POINTER(C.c_float) * 6)(*([C.cast(h.data_ptr(), C.POINTER(C.c_float)) for h in outE] + [None] * 3))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    abi.check(g.lib.fdtd_set_fields_f32(g.h, abi.EH, ptrs), "fdtd_set_fields_f32")
    g.step_graph(K, chunk=GRAPH_CHUNK)
    pr = g.probes()
    abi.check(g.lib.fdtd_get_fields_f32(g.h, abi.E_ALL, optrs), "fdtd_get_fields_f32")
    g.sync()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    h2d = 6 * scene.ncells * 4
    d2h = 3 * scene.ncells * 4 + pr.nbytes
    e2e = {"value": whole_job_gcells(scene.ncells, K, world, e2e_s), "unit": UNIT,
           "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
           "job": "upload 6 fields f32 from pinned host, K steps (fdtd_step_graph), read probes + final E (f32) "
                  "to pinned host"}
    g.close()
    barrier()

    ext = None
    if rank == 0 and world == 1 and not a.no_extensions:
        ext = extensions(a, local)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, thr, kind, n = cpu_sample_run(budget_s=a.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": kind,
               "sample": f"{SAMPLE_DESC}, {n} steps after 1 warm-up, all host threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded Gaussian-correlated height map)",
            "config": config_block(a.res, scene), "clocks": clocks, "e2e": e2e,
            "gpu_launches": gpu_launches, "roofline": roofline,
            "step_roofline": step_roof, "step_roofline_frac": step_roof["frac"],
            "kernels": kernels,
            "farfield_finalize_ms": ff_ms,
            "farfield_points": int(spec.shape[0]),
            "extensions": ext,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def timed_steps(g, K, W, stream):
    """Device time (ms) of K steps of solver g on `stream` after W warm-up steps."""
    import torch
    g.set_stream(stream.cuda_stream)
    g.step(W)
    g.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    g.step(K)
    e1.record(stream)
    torch.cuda.synchronize()
    g.sync()
    return e0.elapsed_time(e1)


def storage_measure(res, storage, K, W, device):
    """Gcell-updates/s of the rough-surface workload with 16-bit field storage."""
    import torch
    from gsvit_copy_b200.solver import Solver
    scene = workload_scene(res, max(4000, K + W + 64))
    scene.storage = storage
    stream = torch.cuda.Stream()
    g = Solver(scene, device=device)
    ms = timed_steps(g, K, W, stream)
    g.close()
    return scene.ncells * K / (ms * 1e-3) / 1e9, ms / K


def batched_measure(K, W, nscenes=48, tune_steps=2):
    """The batched instances (plan.batch_scenes) stepped as one batch from CUDA
    graphs after the tuner picked the bulk work list; device-synchronised host
    clock around K steps."""
    import torch
    from gsvit_copy_b200 import plan
    from gsvit_copy_b200.solver import Batch
    scenes = plan.batch_scenes(nscenes, nsteps=max(2000, K + W + 64))
    cells = sum(sc.ncells for sc in scenes)
    batch = Batch(scenes)
    tune = batch.tune(trial_steps=tune_steps)
    cfg = batch.config()
    batch.step_graph(W + (W % 2), chunk=16)
    batch.sync()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.step_graph(K, chunk=16)
    batch.sync()
    dt = time.perf_counter() - t0
    batch.close()
    return cells, cells * K / dt / 1e9, dt / K * 1e3, cfg, tune


def extensions(a, device):
    """Figures of the library's extensions beyond GSvit's FP32 path, on this
    box, each a separate short run after the headline (not part of `value`):
    the same workload with FP16 and BF16 field storage, and 48 uneven
    instances stepped as one batch."""
    from gsvit_copy_b200 import abi
    K, W = a.ext_steps, 3
    out = {}
    for name, st in (("fp16_storage", abi.STORE_F16), ("bf16_storage", abi.STORE_BF16)):
        v, msps = storage_measure(a.res, st, K, W, device)
        out[name] = {"value": v, "unit": UNIT, "ms_per_step": msps, "steps": K, "warmup": W,
                     "workload": f"rough Drude-silver surface {a.res}^3 (as the headline), {name[:4].upper()} "
                                 "fields / psi / E^n-1 in HBM, FP32 arithmetic"}
    cells, v, msps, cfg, tune = batched_measure(K, W)
    out["batched_48"] = {"value": v, "unit": UNIT, "ms_per_step": msps, "steps": K, "cells": cells,
                         "workload": "48 rough-surface instances, x,y in {64,96,128,192}, z in {64,96,128}, "
                                     "Drude or Lorentz, 8-cell CPML, one batch",
                         "bulk_work_list": cfg, "timing": "host clock around synchronised device work"}
    return out


def run_batched(a):
    """48 independent rough-surface instances (x, y in {64, 96, 128, 192}, z in
    {64, 96, 128}, Drude or Lorentz, 8-cell CPML) stepped as one batch per GPU
    after the autotuner picked its work list, against the same instances
    stepped one by one with the plain solver (each from a CUDA graph).  With N
    ranks (torchrun, one GPU each) the instances are split whole across the
    ranks (plan.shard_instances: no exchange, weak in the instance count per
    GPU), each rank steps its own batch, and the batch arm is timed on the
    device (events on the batch's stream) as the max over ranks.  value =
    the cell updates of all instances over that time."""
    import torch
    from gsvit_copy_b200 import plan
    from gsvit_copy_b200.solver import Batch, Solver
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    ranks = Replicas("nccl", torch.device("cuda", local))
    K, W = a.steps, a.warmup
    scenes_all = plan.batch_scenes(48, nsteps=max(2000, K + W + 64))
    cells_all = [sc.ncells for sc in scenes_all]
    mine = plan.shard_instances(cells_all, world)[rank]
    scenes = [scenes_all[q] for q in mine]
    cells = sum(cells_all)
    batch = Batch(scenes, device=local)
    tune = batch.tune(trial_steps=3)
    cfg = batch.config()
    ext = torch.cuda.ExternalStream(batch.stream_handle())
    batch.step_graph(W + (W % 2), chunk=16)
    batch.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ranks.barrier()
    torch.cuda.synchronize()
    with ClockSampler(bus_id_of(local)) as clk:
        e0.record(ext)
        batch.step_graph(K, chunk=16)
        e1.record(ext)
        torch.cuda.synchronize()
    batch.sync()
    ranks.barrier()
    batch_ms = ranks.max(e0.elapsed_time(e1))
    clocks = clk.summary()
    batch.close()
    # one by one: each instance of this rank its own plan and graph, the same step count
    single_ms = 0.0
    stream = torch.cuda.Stream()
    for sc in scenes:
        g = Solver(sc, device=local)
        g.set_stream(stream.cuda_stream)
        g.step_graph(W + (W % 2), chunk=16)
        g.sync()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        g.step_graph(K, chunk=16)
        f1.record(stream)
        torch.cuda.synchronize()
        g.sync()
        single_ms += f0.elapsed_time(f1)
        g.close()
    single_ms = ranks.max(single_ms)
    value = cells * K / (batch_ms * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": batch_ms / K, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded height maps, sizes, materials, angles)",
            "config": {"workload": "48 rough-surface instances, x,y in {64,96,128,192}, z in {64,96,128}, Drude or Lorentz, "
                                   "8-cell CPML, TSF 0-60 deg, NFFF 3 wavelengths 10x19", "cells": cells,
                       "parallelism": f"instances split whole over {world} GPU(s), no exchange",
                       "instances_rank0": len(mine), "batch_work_list_rank0": cfg,
                       "tuner_rank0": [{"planes_per_item": t[0], "persistent": t[1], "ms_per_step": t[2]} for t in tune]},
            "one_by_one": {"value": cells * K / (single_ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": single_ms / K},
            "speedup_vs_one_by_one": single_ms / batch_ms,
            "timing": "CUDA events on the batch's stream (and the solver stream one by one), max over ranks",
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def run_adjoint(a):
    """The adjoint workload: 256 x 256 x 128 cells of 10 nm, 12-cell CPML,
    4000 steps, a 64 x 64 x 16 design region of per-cell eps_r (seeded
    uniform in [1.5, 4.0]) on a glass slab, 550 nm TSF at normal incidence,
    J = far-field power in a 10 deg cone about theta = 20 deg.  Times the
    forward run alone and the checkpointed gradient (forward, recompute and
    adjoint sweep; checkpoints every 200 steps), and checks --fd-cells seeded
    cells against central differences of J (h = --fd-h on eps_r)."""
    import numpy as np
    from gsvit_copy_b200 import plan
    from gsvit_copy_b200.solver import Solver
    n = a.adj_steps
    s = plan.adjoint_scene(nsteps=n)
    obj = plan.cone_objective(s)
    g = Solver(s)
    init = g.snapshot()
    g.step(1)
    g.sync()
    g.restore(init)
    t0 = time.perf_counter()
    g.step(n)
    g.sync()
    fwd_s = time.perf_counter() - t0
    J0 = g.objective_value(obj)
    # the same forward run replayed from CUDA graphs (captured once before the
    # timed run, bitwise equal to the eager steps), and its per-kernel split
    g.restore(init)
    g.step_graph(100, chunk=50)
    g.sync()
    g.restore(init)
    t0 = time.perf_counter()
    g.step_graph(n, chunk=50)
    g.sync()
    fwd_graph_s = time.perf_counter() - t0
    prof = g.step_profile(8)
    g.restore(init)
    t0 = time.perf_counter()
    J, grad = g.adjoint_gradient(obj, n, 200)
    adj_s = time.perf_counter() - t0
    fd = None
    if a.fd_cells > 0:
        # central differences of J; with --fd-storage f64 through a plan of the
        # same scene with FP64 fields and arithmetic, so that h = 1e-3 is not
        # drowned by FP32 rounding
        from gsvit_copy_b200 import abi
        obj_fd = obj
        if a.fd_storage == "f64":
            s_fd = plan.adjoint_scene(nsteps=n)
            obj_fd = plan.cone_objective(s_fd)   # the same far points, appended to this scene's NFFF
            s_fd.storage = abi.STORE_F64
            g.close()
            g = Solver(s_fd)
        init = g.snapshot()
        g.step(n)
        J_fd = g.objective_value(obj_fd)
        rng = np.random.default_rng(16)
        cells = [tuple(int(rng.integers(0, m)) for m in grad.shape) for _ in range(a.fd_cells)]
        eps0 = s.design["eps"].copy()
        vals = []
        for q in cells:
            jj = []
            for sgn in (1, -1):
                e = eps0.copy()
                e[q] += sgn * a.fd_h
                g.restore(init)
                g.set_design_eps(e)
                g.step(n)
                jj.append(g.objective_value(obj_fd))
            vals.append((jj[0] - jj[1]) / (2 * a.fd_h))
        g.set_design_eps(eps0)
        fdv = np.array(vals)
        adv = np.array([grad[q] for q in cells])
        fd = {"cells": len(cells), "h": a.fd_h, "storage": a.fd_storage, "J_fd_plan": J_fd,
              "max_err_over_max_grad": float(np.abs(adv - fdv).max() / np.abs(grad).max()),
              "max_rel_err": float((np.abs(adv - fdv) / np.abs(adv)).max()),
              "adjoint": adv.tolist(), "finite_differences": fdv.tolist()}
    line = {
        "metric": METRIC, "value": s.ncells * n / fwd_graph_s / 1e9, "unit": UNIT, "n_gpus": 1, "steps": n,
        "warmup": 1, "ms_per_step": fwd_graph_s / n * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "value_is": "forward run replayed from CUDA graphs (fdtd_step_graph)",
        "dtype": "f32", "data": "synthetic (seeded design permittivities)",
        "config": {"workload": "adjoint: 256x256x128 cells 10 nm, 12-cell CPML, 64x64x16 design cells eps_r U[1.5,4] on "
                               "glass eps_r 2.1, 550 nm TSF normal incidence, J = far-field power in a 10 deg cone "
                               "about theta 20 deg, checkpoints every 200 steps", "cells": s.ncells,
                   "design_cells": int(grad.size), "cone_points": int(len(obj["points"]))},
        "forward_graph_s": fwd_graph_s, "forward_eager_s": fwd_s, "forward_eager_gcells": s.ncells * n / fwd_s / 1e9,
        "kernel_ms_per_step": {k: prof[k] / 8 for k in ("bulk_ms", "slab_ms", "aux_ms", "nfff_ms", "total_ms")},
        "adjoint": {"J": J, "J_forward_only": J0, "forward_s": fwd_s, "gradient_s": adj_s, "gradient_over_forward": adj_s / fwd_s,
                    "grad_min": float(grad.min()), "grad_max": float(grad.max()), "fd": fd},
        "timing": "host clock around synchronised device work",
    }
    print(json.dumps(line), flush=True)
    return 0


def _rel(a, b, chunk=1 << 24):
    """Relative L2 distance |a - b| / |b| of two large arrays, in chunks (no full-size temporaries)."""
    import numpy as np
    a, b = a.reshape(-1), b.reshape(-1)
    num = den = 0.0
    for q in range(0, b.size, chunk):
        x = a[q:q + chunk].astype(np.float64)
        y = b[q:q + chunk].astype(np.float64)
        num += float(np.dot(x - y, x - y))
        den += float(np.dot(y, y))
    return (num / den) ** 0.5 if den > 0 else num ** 0.5


def run_precision(a):
    """The FP64 pin of the headline workload at full size: the 512^3 rough
    Drude-silver surface stepped --prec-steps steps with FP64 field storage and
    arithmetic (FDTD_STORE_F64: the reference's own precision), then with FP32,
    FP16 and BF16 storage; E, the probe series and the far-field spectrum of
    each against the FP64 run (relative L2), and each run's device time."""
    import numpy as np
    import torch
    from gsvit_copy_b200 import abi
    from gsvit_copy_b200.solver import Solver
    n = a.prec_steps
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    runs = {}
    ref = None
    for name, st in (("f64", abi.STORE_F64), ("f32", abi.STORE_F32), ("f16", abi.STORE_F16), ("bf16", abi.STORE_BF16)):
        scene = workload_scene(a.res, n)
        scene.storage = st
        cfg = config_block(a.res, scene)
        g = Solver(scene, device=0)
        g.set_stream(stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        g.step(n)
        e1.record(stream)
        torch.cuda.synchronize()
        g.sync()
        ms = e0.elapsed_time(e1)
        E = g.fields(abi.E_ALL, dtype=np.float32 if st != abi.STORE_F64 else np.float64)[:3]
        out = {"gcells": scene.ncells * n / (ms * 1e-3) / 1e9, "ms_per_step": ms / n,
               "probes": g.probes(), "spectrum": g.nfff_spectrum(), "E": E}
        g.close()
        if ref is None:
            ref = out
            runs[name] = {"value": out["gcells"], "ms_per_step": out["ms_per_step"]}
            continue
        runs[name] = {"value": out["gcells"], "ms_per_step": out["ms_per_step"],
                      "rel_l2_E": [_rel(x, y) for x, y in zip(out["E"], ref["E"])],
                      "rel_l2_probes": _rel(out["probes"], ref["probes"]),
                      "rel_l2_farfield": _rel(out["spectrum"], ref["spectrum"])}
        del out
    line = {
        "metric": METRIC, "value": runs["f32"]["value"], "unit": UNIT, "n_gpus": 1, "steps": n, "warmup": 0,
        "ms_per_step": runs["f32"]["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Gaussian-correlated height map)",
        "config": dict(cfg, workload_kind="precision pin against FP64"),
        "precision": runs,
        "tolerance_note": "rel L2 of E, probe series and far-field spectrum after the full run, against the FP64 run",
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.workload == "precision":
        return run_precision(a)
    if a.workload == "batched":
        return run_batched(a)
    if a.workload == "adjoint":
        return run_adjoint(a)
    if a.impl == "reference":
        return run_reference(a)
    return run_b200(a)


if __name__ == "__main__":
    sys.exit(main())
