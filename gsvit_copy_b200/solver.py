"""Python host mirror of the C ABI: one `Solver` per plan.

The method names follow the stages of GSvit's GPU driver they replace
(sv_pool_gpu_copyto / copyfrom / ystep_* / getpoints / apply_farfield,
pool.h:98-128); the work itself runs in libgsvit_b200.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import abi


class Solver:
    def __init__(self, scene, device: int = 0, _handle=None):
        self.lib = abi.load_library()
        self.scene = scene
        self.shape = (scene.xres, scene.yres, scene.zres)
        self.n = scene.ncells
        self._owner = _handle is None
        if _handle is not None:     # a plan owned by a Batch
            self.h = _handle
            return
        self._desc, self._keep = scene.desc()
        h = C.c_void_p()
        abi.check(self.lib.fdtd_plan_create(C.byref(self._desc), device, C.byref(h)), "fdtd_plan_create")
        self.h = h

    # -- lifetime
    def close(self):
        if getattr(self, "h", None) and self._owner:
            self.lib.fdtd_plan_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle: Optional[int]):
        abi.check(self.lib.fdtd_set_stream(self.h, C.c_void_p(stream_handle or 0)), "fdtd_set_stream")

    def sync(self):
        abi.check(self.lib.fdtd_sync(self.h), "fdtd_sync")

    # -- fields (sv_pool_gpu_copyto / copyfrom)
    def set_fields(self, comps: Sequence[Optional[np.ndarray]], mask: int = abi.EH):
        arrs = [None if c is None else np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in comps]
        abi.check(self.lib.fdtd_set_fields(self.h, mask, abi.field_ptrs(arrs)), "fdtd_set_fields")

    def fields(self, mask: int = abi.EH, dtype=np.float64):
        if dtype == np.float32:
            out = [np.empty(self.shape, dtype=np.float32) if mask & (1 << c) else None for c in range(6)]
            abi.check(self.lib.fdtd_get_fields_f32(self.h, mask, abi.field_ptrs(out, C.c_float)), "fdtd_get_fields_f32")
        else:
            out = [np.empty(self.shape) if mask & (1 << c) else None for c in range(6)]
            abi.check(self.lib.fdtd_get_fields(self.h, mask, abi.field_ptrs(out)), "fdtd_get_fields")
        return out

    # -- stepping
    def step(self, n: int = 1):
        abi.check(self.lib.fdtd_step(self.h, n), "fdtd_step")

    def step_graph(self, n: int, chunk: int = 32):
        abi.check(self.lib.fdtd_step_graph(self.h, n, chunk), "fdtd_step_graph")

    def step_timed(self, n: int):
        ms = C.c_double()
        cnt = C.c_int()
        abi.check(self.lib.fdtd_step_timed(self.h, n, C.byref(ms), C.byref(cnt)), "fdtd_step_timed")
        return ms.value, cnt.value

    def step_profile(self, n: int) -> dict:
        out = (C.c_double * 8)()
        abi.check(self.lib.fdtd_step_profile(self.h, n, out), "fdtd_step_profile")
        keys = ["bulk_ms", "bulk_bytes", "slab_ms", "slab_bytes", "aux_ms", "nfff_ms", "total_ms", "launches_per_step"]
        return dict(zip(keys, list(out)))

    @property
    def step_count(self) -> int:
        s = C.c_int()
        abi.check(self.lib.fdtd_get_step(self.h, C.byref(s)), "fdtd_get_step")
        return s.value

    # -- outputs
    def probes(self) -> np.ndarray:
        p = 0 if self.scene.probes is None else len(self.scene.probes)
        out = np.zeros((p, max(self.scene.nsteps, 1), 6))
        if p:
            abi.check(self.lib.fdtd_get_probes(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size),
                      "fdtd_get_probes")
        return out

    def nfff_spectrum(self) -> np.ndarray:
        """Complex far-field DFT, shape (npoints, nfreq, 3)."""
        f = self.scene.nfff
        npt, nf = len(f["points"]), len(f["omega"])
        out = np.zeros((npt, nf, 3, 2))
        abi.check(self.lib.fdtd_nfff_spectrum(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size),
                  "fdtd_nfff_spectrum")
        return out[..., 0] + 1j * out[..., 1]

    def nfff_series(self) -> np.ndarray:
        """Time-domain far-field series (npoints, 3, ndata) of a plan with nfff["series"]."""
        nd = C.c_int()
        abi.check(self.lib.fdtd_nfff_ndata(self.h, C.byref(nd)), "fdtd_nfff_ndata")
        npt = len(self.scene.nfff["points"])
        out = np.zeros((npt, 3, nd.value))
        abi.check(self.lib.fdtd_nfff_series(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size),
                  "fdtd_nfff_series")
        return out

    def map(self, which: int) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.int32)
        abi.check(self.lib.fdtd_get_map(self.h, which, out.ctypes.data_as(C.POINTER(C.c_int32)), out.size),
                  "fdtd_get_map")
        return out

    @property
    def nclasses(self) -> int:
        v = C.c_int()
        abi.check(self.lib.fdtd_get_nclasses(self.h, C.byref(v)), "fdtd_get_nclasses")
        return v.value

    def step_bytes(self) -> float:
        v = C.c_double()
        abi.check(self.lib.fdtd_step_bytes(self.h, C.byref(v)), "fdtd_step_bytes")
        return v.value

    # -- checkpoints
    def snapshot(self) -> bytearray:
        sz = C.c_size_t()
        abi.check(self.lib.fdtd_snapshot_size(self.h, C.byref(sz)), "fdtd_snapshot_size")
        buf = bytearray(sz.value)
        cbuf = (C.c_char * sz.value).from_buffer(buf)
        abi.check(self.lib.fdtd_snapshot_save(self.h, C.cast(cbuf, C.c_void_p), sz.value), "fdtd_snapshot_save")
        return buf

    def restore(self, buf: bytearray):
        cbuf = (C.c_char * len(buf)).from_buffer(buf)
        abi.check(self.lib.fdtd_snapshot_restore(self.h, C.cast(cbuf, C.c_void_p), len(buf)), "fdtd_snapshot_restore")

    # -- adjoint (design region, far-field objective)
    def set_design_eps(self, eps: np.ndarray):
        """New relative permittivities of the design cells (shape of the box)."""
        e = np.ascontiguousarray(eps, dtype=np.float64).reshape(-1)
        abi.check(self.lib.fdtd_set_design_eps(self.h, e.ctypes.data_as(C.POINTER(C.c_double))), "fdtd_set_design_eps")
        self.scene.design = dict(self.scene.design, eps=np.array(eps, dtype=np.float64).reshape(self._design_shape()))

    def _design_shape(self):
        i0, i1, j0, j1, k0, k1 = self.scene.design["box"]
        return (i1 - i0, j1 - j0, k1 - k0)

    @staticmethod
    def _objective(obj: dict):
        pts = np.ascontiguousarray(obj["points"], dtype=np.int32)
        w = np.ascontiguousarray(obj["weights"], dtype=np.float64)
        o = abi.Objective(freq=int(obj.get("freq", 0)), npoints=len(pts), points=abi.as_ptr(pts, C.c_int32),
                          weights=abi.as_ptr(w, C.c_double))
        return o, (pts, w)

    def objective_value(self, obj: dict) -> float:
        """J = sum_t w_t |F(p_t)|^2 of the far field accumulated so far."""
        o, keep = self._objective(obj)
        J = C.c_double()
        abi.check(self.lib.fdtd_objective_value(self.h, C.byref(o), C.byref(J)), "fdtd_objective_value")
        return J.value

    def adjoint_gradient(self, obj: dict, nsteps: int, checkpoint: int = 200):
        """Forward nsteps (checkpointed), J, and dJ/d eps_r of the design cells
        by the discrete adjoint; returns (J, grad with the design box shape)."""
        o, keep = self._objective(obj)
        J = C.c_double()
        grad = np.zeros(self._design_shape())
        abi.check(self.lib.fdtd_adjoint_gradient(self.h, C.byref(o), nsteps, checkpoint, C.byref(J),
                                                 grad.ctypes.data_as(C.POINTER(C.c_double))), "fdtd_adjoint_gradient")
        return J.value, grad

    def adjoint_transpose(self, comps: Sequence[np.ndarray], nsteps: int):
        """The transposed step applied nsteps times to an adjoint state (E then
        H components); returns the six new components."""
        arrs = [np.ascontiguousarray(c, dtype=np.float64).copy() for c in comps]
        ptrs = (C.POINTER(C.c_double) * 6)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        abi.check(self.lib.fdtd_adjoint_transpose(self.h, nsteps, ptrs), "fdtd_adjoint_transpose")
        return arrs


class Batch:
    """Many scenes stepped in lockstep, one launch per kernel for all of them
    (fdtd_batch_*).  `batch[i]` is a Solver view of instance i for fields,
    probes, far fields and maps; step through the batch only."""

    def __init__(self, scenes, device: int = 0):
        self.lib = abi.load_library()
        self.scenes = list(scenes)
        descs, self._keep = [], []
        for sc in self.scenes:
            d, k = sc.desc()
            descs.append(d)
            self._keep.append(k)
        self._descs = (abi.Desc * len(descs))(*descs)
        h = C.c_void_p()
        abi.check(self.lib.fdtd_batch_create(self._descs, len(descs), device, C.byref(h)), "fdtd_batch_create")
        self.h = h
        self.views = []
        for i, sc in enumerate(self.scenes):
            ph = C.c_void_p()
            abi.check(self.lib.fdtd_batch_plan(self.h, i, C.byref(ph)), "fdtd_batch_plan")
            self.views.append(Solver(sc, _handle=ph))

    def __len__(self):
        return len(self.views)

    def __getitem__(self, i):
        return self.views[i]

    def close(self):
        if getattr(self, "h", None):
            for v in self.views:
                v.h = None
            self.lib.fdtd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        abi.check(self.lib.fdtd_batch_step(self.h, n), "fdtd_batch_step")

    def step_graph(self, n: int, chunk: int = 16):
        abi.check(self.lib.fdtd_batch_step_graph(self.h, n, chunk), "fdtd_batch_step_graph")

    def sync(self):
        abi.check(self.lib.fdtd_batch_sync(self.h), "fdtd_batch_sync")

    def stream_handle(self) -> int:
        """The batch's CUDA stream (cudaStream_t as an integer), e.g. for
        torch.cuda.ExternalStream and events around its steps."""
        p = C.c_void_p()
        abi.check(self.lib.fdtd_batch_get_stream(self.h, C.byref(p)), "fdtd_batch_get_stream")
        return p.value or 0

    def tune(self, trial_steps: int = 4):
        """Autotune the work list; returns [(planes per item (0 = whole), persistent, ms/step), ...]."""
        rep = (C.c_double * 60)()
        n = C.c_int()
        abi.check(self.lib.fdtd_batch_tune(self.h, trial_steps, rep, 60, C.byref(n)), "fdtd_batch_tune")
        return [(int(rep[3 * i]), bool(rep[3 * i + 1]), rep[3 * i + 2]) for i in range(n.value)]

    def config(self) -> dict:
        v = [C.c_int() for _ in range(4)]
        abi.check(self.lib.fdtd_batch_config(self.h, *[C.byref(x) for x in v]), "fdtd_batch_config")
        return dict(zip(["planes_per_item", "persistent", "grid", "items"], [x.value for x in v]))
