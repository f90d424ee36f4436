"""ctypes wrapper of the FP64 CPU restatement (oracle/fdtd_oracle.c) and of the
reference CPU solver built from GSvit's own sources (oracle/_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgsvit_ref.so")


def build_oracle(force: bool = False) -> str:
    """Compile the restatement (gcc, OpenMP) if it is not built yet."""
    src = os.path.join(HERE, "fdtd_oracle.c")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", ORACLE_SO, src, "-lm"])
    return ORACLE_SO


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _bind(lib, prefix):
    P = C.c_void_p
    sig = {
        "create": ([P, C.c_char_p], P),
        "destroy": ([P], None),
        "step": ([P, C.c_int], C.c_int),
        "get_fields": ([P] + [_dp] * 6, C.c_int),
        "set_fields": ([P] + [_dp] * 6, C.c_int),
        "get_map": ([P, C.c_int, _ip], C.c_int),
        "get_probes": ([P, _dp], C.c_int),
        "nfff_ndata": ([P], C.c_int),
        "get_nfff_series": ([P, _dp], C.c_int),
        "get_nfff_istart": ([P, _ip], C.c_int),
        "aux_res": ([P], C.c_int),
        "get_aux": ([P, _dp, _dp], C.c_int),
        "get_step": ([P], C.c_int),
    }
    for k, (a, r) in sig.items():
        fn = getattr(lib, prefix + k)
        fn.argtypes = a
        fn.restype = r
    return lib


_LIBS = {}


def _load(kind: str):
    if kind in _LIBS:
        return _LIBS[kind]
    if kind == "oracle":
        lib = _bind(C.CDLL(build_oracle()), "oracle_")
    else:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        lib = _bind(C.CDLL(REF_SO), "ref_")
    _LIBS[kind] = (lib, "oracle_" if kind == "oracle" else "ref_")
    return _LIBS[kind]


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class CpuSolver:
    """One FP64 CPU run of a Scene: kind 'oracle' (restatement) or 'reference'
    (GSvit's own yee.c/boundary.c/source.c/... built under oracle/_ref)."""

    def __init__(self, scene, kind: str = "oracle"):
        self.lib, self.pre = _load(kind)
        self.scene = scene
        self._desc, self._keep = scene.desc()
        err = C.create_string_buffer(256)
        self.h = self._f("create")(C.byref(self._desc), err)
        if not self.h:
            raise RuntimeError(f"{kind} create failed: {err.value.decode()}")
        self.n = scene.ncells
        self.shape = (scene.xres, scene.yres, scene.zres)

    def _f(self, name):
        return getattr(self.lib, self.pre + name)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int):
        rc = self._f("step")(self.h, n)
        if rc != 0:
            raise RuntimeError(f"step rc={rc}")

    @property
    def step_count(self) -> int:
        return self._f("get_step")(self.h)

    def fields(self):
        out = [np.empty(self.shape) for _ in range(6)]
        self._f("get_fields")(self.h, *[o.ctypes.data_as(_dp) for o in out])
        return out

    def set_fields(self, comps):
        arrs = [np.ascontiguousarray(c, dtype=np.float64) for c in comps]
        self._f("set_fields")(self.h, *[a.ctypes.data_as(_dp) for a in arrs])

    def map(self, which: int):
        out = np.empty(self.shape, dtype=np.int32)
        rc = self._f("get_map")(self.h, which, out.ctypes.data_as(_ip))
        if rc != 0:
            raise RuntimeError("get_map")
        return out

    def probes(self):
        p = len(self.scene.probes) if self.scene.probes is not None else 0
        out = np.zeros((p, self.scene.nsteps, 6))
        if p:
            self._f("get_probes")(self.h, out.ctypes.data_as(_dp))
        return out

    def nfff_series(self):
        nd = self._f("nfff_ndata")(self.h)
        npt = len(self.scene.nfff["points"])
        out = np.zeros((npt, 3, nd))
        self._f("get_nfff_series")(self.h, out.ctypes.data_as(_dp))
        return out

    def nfff_istart(self):
        npt = len(self.scene.nfff["points"])
        out = np.zeros(npt, dtype=np.int32)
        self._f("get_nfff_istart")(self.h, out.ctypes.data_as(_ip))
        return out

    def aux(self):
        r = self._f("aux_res")(self.h)
        e = np.zeros(r)
        h = np.zeros(r)
        if r:
            self._f("get_aux")(self.h, e.ctypes.data_as(_dp), h.ctypes.data_as(_dp))
        return e, h


def series_spectrum(series: np.ndarray, omega: np.ndarray, dt: float) -> np.ndarray:
    """DFT sum_m F[m] exp(-i w m dt) of reference far-field series
    (npoints, 3, ndata) at the angular frequencies omega -> (npoints, nfreq, 3)."""
    m = np.arange(series.shape[-1])
    ph = np.exp(-1j * np.outer(omega, m) * dt)            # (nfreq, ndata)
    return np.einsum("pcm,fm->pfc", series, ph)
