"""GSvit's own CUDA path (src3d/gpu.c + gpu_kernels.cu, compiled unmodified
for sm_100a into oracle/_ref/libgsvit_refcuda.so) stepped through the GPU
branch of svit.c:240-256, timed on the host clock.

TEST INFRASTRUCTURE ONLY: the measured context baseline of bench.py's
reference arm and of the tests.  The product never imports it.

The reference runs one worker thread per device that spins on a task queue
until the process exits (gpu.c:1792-1955), and every stage ends in a device
synchronisation (the wrap_* functions of gpu_kernels.cu), so the host clock
around K steps is the device time of K steps.  `run()` starts a child process
(`python -m oracle.refcuda ...`) that prints one JSON line, so the caller's
process holds no second CUDA context and no spinning thread.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REFCUDA_SO = os.path.join(HERE, "_ref", "libgsvit_refcuda.so")
_dp = C.POINTER(C.c_double)


def available() -> bool:
    return os.path.exists(REFCUDA_SO)


def _lib():
    lib = C.CDLL(REFCUDA_SO)
    P = C.c_void_p
    for name, a, r in [("ref_create", [P, C.c_char_p], P), ("ref_get_fields", [P] + [_dp] * 6, C.c_int),
                       ("ref_set_fields", [P] + [_dp] * 6, C.c_int), ("ref_nfff_ndata", [P], C.c_int),
                       ("ref_get_nfff_series", [P, _dp], C.c_int), ("dropin_start", [P], C.c_int),
                       ("dropin_step", [P, C.c_int], C.c_int), ("dropin_finish", [P], C.c_int),
                       ("dropin_get_probes", [P, _dp], C.c_int)]:
        f = getattr(lib, name)
        f.argtypes, f.restype = a, r
    return lib


def _scene(kind: str, res: int, nsteps: int, nfff: bool, angles):
    sys.path.insert(0, ROOT)
    from gsvit_copy_b200 import plan
    if kind == "rough":
        return plan.rough_surface_scene(res=res, nsteps=nsteps, nfff_angles=tuple(angles) if nfff else None)
    if kind == "vacuum":
        # the small scene's CPML, TSF, NFFF and probes without its materials
        s = plan.small_scene("lintab", shape=(res, res + 8, res + 24), nsteps=nsteps)
        s.mat[:] = 0
        return s
    return plan.small_scene(kind, shape=(res, res + 8, res + 24), nsteps=nsteps)


def measure(kind: str, res: int, steps: int, warmup: int, nfff: bool = True, angles=(91, 181), fields_in=None,
            out_npz=None) -> dict:
    """In this process: build the scene, set the six fields from `fields_in`
    (an .npz of arr_0 .. arr_5, FP64) if given, create the reference's GPU
    plan (sv_gpu_new, gpu_init, copyto), run `warmup` steps, time `steps`
    steps, copy the fields back (optionally to `out_npz`, arr_0 .. arr_5)."""
    lib = _lib()
    s = _scene(kind, res, warmup + steps + 2, nfff, angles)
    desc, keep = s.desc()
    err = C.create_string_buffer(256)
    t0 = time.perf_counter()
    h = lib.ref_create(C.byref(desc), err)
    if not h:
        raise RuntimeError(err.value.decode())
    shape = (s.xres, s.yres, s.zres)
    if fields_in:
        z = np.load(fields_in)
        comps = [np.ascontiguousarray(z[f"arr_{c}"], dtype=np.float64) for c in range(6)]
        assert all(c.shape == shape for c in comps), "field shape"
        lib.ref_set_fields(h, *[a.ctypes.data_as(_dp) for a in comps])
    t1 = time.perf_counter()
    if lib.dropin_start(h) != 0:
        raise RuntimeError("sv_gpu_new / gpu_init / copyto failed")
    t2 = time.perf_counter()
    if warmup and lib.dropin_step(h, warmup) != 0:
        raise RuntimeError("reference GPU step failed")
    t3 = time.perf_counter()
    if lib.dropin_step(h, steps) != 0:
        raise RuntimeError("reference GPU step failed")
    t4 = time.perf_counter()
    if lib.dropin_finish(h) != 0:
        raise RuntimeError("reference copyfrom failed")
    out = [np.empty(shape) for _ in range(6)]
    lib.ref_get_fields(h, *[o.ctypes.data_as(_dp) for o in out])
    finite = bool(all(np.isfinite(o).all() for o in out))
    if out_npz:
        np.savez(out_npz, *out)
    cells = s.xres * s.yres * s.zres
    sec = t4 - t3
    return {"kind": kind, "shape": list(shape), "cells": cells, "steps": steps, "warmup": warmup,
            "nfff_points": int(len(s.nfff["points"])) if (nfff and s.nfff) else 0,
            "seconds": sec, "ms_per_step": sec / steps * 1e3, "gcells": cells * steps / sec / 1e9,
            "setup_s": t1 - t0, "gpu_setup_s": t2 - t1, "warmup_s": t3 - t2, "finite": finite,
            "max_abs_e": float(max(np.abs(o).max() for o in out[:3]))}


def run(kind: str = "rough", res: int = 128, steps: int = 10, warmup: int = 2, nfff: bool = True, angles=(91, 181),
        fields_in=None, out_npz=None, timeout: float = 900.0) -> dict:
    """`measure` in a child process; returns its JSON line as a dict."""
    cmd = [sys.executable, "-m", "oracle.refcuda", "--kind", kind, "--res", str(res), "--steps", str(steps),
           "--warmup", str(warmup), "--angles", str(angles[0]), str(angles[1])]
    if not nfff:
        cmd.append("--no-nfff")
    if fields_in:
        cmd += ["--fields-in", fields_in]
    if out_npz:
        cmd += ["--out", out_npz]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    if p.returncode != 0 or not lines:
        raise RuntimeError(f"reference CUDA run failed (rc {p.returncode}): {(p.stderr or p.stdout)[-1500:]}")
    return json.loads(lines[-1])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kind", default="rough")
    ap.add_argument("--res", type=int, default=128)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--angles", type=int, nargs=2, default=(91, 181))
    ap.add_argument("--no-nfff", action="store_true")
    ap.add_argument("--fields-in", default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    d = measure(a.kind, a.res, a.steps, a.warmup, not a.no_nfff, a.angles, a.fields_in, a.out)
    # on a line of its own: the reference's unterminated printf output may precede it
    print("\n" + json.dumps(d), flush=True)
    # the reference's worker thread never returns: end the process here
    os._exit(0)


if __name__ == "__main__":
    main()
