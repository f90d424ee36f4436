"""GSvit's own CPU code with its GPU branch stepped through the drop-in
(gsvit_copy_b200/dropin/gpu_b200.c over libgsvit_b200), loaded from
oracle/_ref/libgsvit_dropin.so.  Test helper only."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN_SO = os.path.join(ROOT, "oracle", "_ref", "libgsvit_dropin.so")
_dp = C.POINTER(C.c_double)
_LIB = None


def available() -> bool:
    return os.path.exists(DROPIN_SO)


def _lib():
    global _LIB
    if _LIB is None:
        lib = C.CDLL(DROPIN_SO)
        P = C.c_void_p
        for name, a, r in [("ref_create", [P, C.c_char_p], P), ("ref_step", [P, C.c_int], C.c_int),
                           ("ref_get_fields", [P] + [_dp] * 6, C.c_int), ("ref_set_fields", [P] + [_dp] * 6, C.c_int),
                           ("ref_nfff_ndata", [P], C.c_int), ("ref_get_nfff_series", [P, _dp], C.c_int),
                           ("ref_get_probes", [P, _dp], C.c_int), ("dropin_start", [P], C.c_int),
                           ("dropin_step", [P, C.c_int], C.c_int), ("dropin_finish", [P], C.c_int),
                           ("dropin_get_probes", [P, _dp], C.c_int), ("dropin_request", [P, C.c_int], C.c_int)]:
            f = getattr(lib, name)
            f.argtypes, f.restype = a, r
        _LIB = lib
    return _LIB


class DropinRun:
    """One scene through GSvit's structures: `gpu=False` steps the CPU branch of
    svit.c, `gpu=True` the GPU branch (sv_pool_gpu_*) through the drop-in."""

    def __init__(self, scene, gpu: bool):
        self.lib = _lib()
        self.scene = scene
        self.gpu = gpu
        self._desc, self._keep = scene.desc()
        err = C.create_string_buffer(256)
        self.h = self.lib.ref_create(C.byref(self._desc), err)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.shape = (scene.xres, scene.yres, scene.zres)
        self.started = False

    def set_fields(self, comps):
        arrs = [np.ascontiguousarray(c, dtype=np.float64) for c in comps]
        self.lib.ref_set_fields(self.h, *[a.ctypes.data_as(_dp) for a in arrs])

    def step(self, n):
        if self.gpu:
            if not self.started:
                assert self.lib.dropin_start(self.h) == 0
                self.started = True
            assert self.lib.dropin_step(self.h, n) == 0
        else:
            assert self.lib.ref_step(self.h, n) == 0

    def finish(self):
        if self.gpu:
            assert self.lib.dropin_finish(self.h) == 0

    def fields(self):
        out = [np.empty(self.shape) for _ in range(6)]
        self.lib.ref_get_fields(self.h, *[o.ctypes.data_as(_dp) for o in out])
        return out

    def probes(self):
        p = len(self.scene.probes)
        out = np.zeros((p, self.scene.nsteps, 6))
        (self.lib.dropin_get_probes if self.gpu else self.lib.ref_get_probes)(self.h, out.ctypes.data_as(_dp))
        return out

    def nfff_series(self):
        nd = self.lib.ref_nfff_ndata(self.h)
        out = np.zeros((len(self.scene.nfff["points"]), 3, nd))
        self.lib.ref_get_nfff_series(self.h, out.ctypes.data_as(_dp))
        return out
