"""ctypes mirror of include/gsvit_b200.h and the loader of the CUDA library.

The structures below are field-for-field copies of the C declarations; the
library itself (gsvit_copy_b200/libgsvit_b200.so) is built by
gsvit_copy_b200/build.py.  There is no fallback: if the shared library is
missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ABI_VERSION = 2

OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "unsupported",
    -3: "CUDA error",
    -4: "out of memory",
    -5: "bad state",
    -6: "timeout",
}

MAT_LINEAR, MAT_LINTAB, MAT_DRUDE, MAT_CP3, MAT_CP, MAT_ADE, MAT_PLRC, MAT_PEC = 0, 1, 2, 3, 4, 5, 6, 10
MATMODE_NONE, MATMODE_ELECTRIC, MATMODE_MAGNETIC, MATMODE_FULL = 0, 1, 2, 3
FACE_X0, FACE_XN, FACE_Y0, FACE_YN, FACE_Z0, FACE_ZN = range(6)
STORE_F32, STORE_F16, STORE_BF16, STORE_F64 = 0, 1, 2, 3
EX, EY, EZ, HX, HY, HZ = 0x01, 0x02, 0x04, 0x08, 0x10, 0x20
E_ALL, H_ALL = EX | EY | EZ, HX | HY | HZ
EH = E_ALL | H_ALL
MAP_MAT, MAP_BNDS, MAP_SOURCESKIP, MAP_CLASS = 0, 1, 2, 3
STATIC_SCRATCH_BYTES = 32 * 1024 * 1024

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class Material(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("reserved", C.c_int32),
        ("epsilon", C.c_double), ("mu", C.c_double), ("sigma", C.c_double), ("sigast", C.c_double),
        ("drude_omega_p", C.c_double), ("drude_nu", C.c_double),
        ("cp_a", C.c_double * 2), ("cp_phi", C.c_double * 2),
        ("cp_omega", C.c_double * 2), ("cp_gamma", C.c_double * 2),
        ("ade_a0", C.c_double), ("ade_a1", C.c_double), ("ade_a2", C.c_double),
        ("ade_bp0", C.c_double * 2), ("ade_bp1", C.c_double * 2), ("ade_bp2", C.c_double * 2),
        ("ade_bp3", C.c_double * 2), ("ade_bp4", C.c_double * 2),
        ("ade_c0", C.c_double), ("ade_c1", C.c_double), ("ade_c2", C.c_double), ("ade_c3", C.c_double),
    ]


class CpmlFace(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("depth", C.c_int32), ("m", C.c_int32), ("reserved", C.c_int32),
                ("sigma", C.c_double), ("kappa", C.c_double), ("a", C.c_double)]


class Tsf(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("i0", C.c_int32), ("j0", C.c_int32), ("k0", C.c_int32),
        ("in_", C.c_int32), ("jn", C.c_int32), ("kn", C.c_int32),
        ("skip", C.c_int32 * 6), ("skipdepth", C.c_int32),
        ("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double),
        ("layered_epsilon", C.c_double), ("layered_mu", C.c_double),
        ("nwave", C.c_int32), ("reserved", C.c_int32), ("wave", _dp),
    ]


class Nfff(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("i0", C.c_int32), ("j0", C.c_int32), ("k0", C.c_int32),
        ("in_", C.c_int32), ("jn", C.c_int32), ("kn", C.c_int32),
        ("skip", C.c_int32 * 6), ("skip_lo", (C.c_int32 * 2) * 6), ("skip_hi", (C.c_int32 * 2) * 6),
        ("npoints", C.c_int32), ("nfreq", C.c_int32), ("series", C.c_int32), ("reserved", C.c_int32),
        ("points", _ip), ("istart", _ip), ("omega", _dp),
    ]


class Design(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("i0", C.c_int32), ("i1", C.c_int32), ("j0", C.c_int32), ("j1", C.c_int32),
                ("k0", C.c_int32), ("k1", C.c_int32), ("reserved", C.c_int32), ("eps_r", C.POINTER(C.c_double))]


class Objective(C.Structure):
    _fields_ = [("freq", C.c_int32), ("npoints", C.c_int32), ("points", _ip), ("weights", C.POINTER(C.c_double))]


class Desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("xres", C.c_int32), ("yres", C.c_int32), ("zres", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("nsteps", C.c_int32), ("matmode", C.c_int32), ("nmat", C.c_int32), ("storage", C.c_int32),
        ("mats", C.POINTER(Material)), ("mat", _ip),
        ("epsilon", _fp), ("sigma", _fp), ("mu", _fp), ("sigast", _fp),
        ("cpml", CpmlFace * 6), ("tsf", Tsf), ("nfff", Nfff),
        ("nprobes", C.c_int32), ("reserved", C.c_int32), ("probes", _ip),
        ("design", Design),
    ]


def as_ptr(arr, ctype):
    """Pointer to the data of a C-contiguous numpy array (None -> NULL)."""
    if arr is None:
        return C.cast(None, C.POINTER(ctype))
    assert arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(ctype))


_LIB = None
LIB_NAME = "libgsvit_b200.so"


def lib_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)


def load_library():
    """Load the in-tree CUDA library; raise if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m gsvit_copy_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    P = C.c_void_p
    sig = {
        "fdtd_plan_create": ([C.POINTER(Desc), C.c_int, C.POINTER(P)], C.c_int),
        "fdtd_plan_destroy": ([P], C.c_int),
        "fdtd_set_stream": ([P, P], C.c_int),
        "fdtd_sync": ([P], C.c_int),
        "fdtd_set_fields": ([P, C.c_int, C.POINTER(_dp)], C.c_int),
        "fdtd_get_fields": ([P, C.c_int, C.POINTER(_dp)], C.c_int),
        "fdtd_set_fields_f32": ([P, C.c_int, C.POINTER(_fp)], C.c_int),
        "fdtd_get_fields_f32": ([P, C.c_int, C.POINTER(_fp)], C.c_int),
        "fdtd_step": ([P, C.c_int], C.c_int),
        "fdtd_step_graph": ([P, C.c_int, C.c_int], C.c_int),
        "fdtd_step_static_scratch": ([P, C.c_int], C.c_int),
        "fdtd_get_step": ([P, C.POINTER(C.c_int)], C.c_int),
        "fdtd_step_timed": ([P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)], C.c_int),
        "fdtd_step_profile": ([P, C.c_int, _dp], C.c_int),
        "fdtd_get_probes": ([P, _dp, C.c_size_t], C.c_int),
        "fdtd_nfff_spectrum": ([P, _dp, C.c_size_t], C.c_int),
        "fdtd_nfff_ndata": ([P, C.POINTER(C.c_int)], C.c_int),
        "fdtd_nfff_series": ([P, _dp, C.c_size_t], C.c_int),
        "fdtd_get_map": ([P, C.c_int, _ip, C.c_size_t], C.c_int),
        "fdtd_get_nclasses": ([P, C.POINTER(C.c_int)], C.c_int),
        "fdtd_snapshot_size": ([P, C.POINTER(C.c_size_t)], C.c_int),
        "fdtd_snapshot_save": ([P, P, C.c_size_t], C.c_int),
        "fdtd_snapshot_restore": ([P, P, C.c_size_t], C.c_int),
        "fdtd_last_error": ([], C.c_char_p),
        "fdtd_step_bytes": ([P, C.POINTER(C.c_double)], C.c_int),
        "fdtd_batch_create": ([C.POINTER(Desc), C.c_int, C.c_int, C.POINTER(P)], C.c_int),
        "fdtd_batch_destroy": ([P], C.c_int),
        "fdtd_batch_size": ([P, C.POINTER(C.c_int)], C.c_int),
        "fdtd_batch_plan": ([P, C.c_int, C.POINTER(P)], C.c_int),
        "fdtd_batch_step": ([P, C.c_int], C.c_int),
        "fdtd_batch_step_graph": ([P, C.c_int, C.c_int], C.c_int),
        "fdtd_batch_sync": ([P], C.c_int),
        "fdtd_batch_tune": ([P, C.c_int, _dp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "fdtd_batch_config": ([P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "fdtd_batch_get_stream": ([P, C.POINTER(P)], C.c_int),
        "fdtd_set_design_eps": ([P, _dp], C.c_int),
        "fdtd_objective_value": ([P, C.POINTER(Objective), _dp], C.c_int),
        "fdtd_adjoint_gradient": ([P, C.POINTER(Objective), C.c_int, C.c_int, _dp, _dp], C.c_int),
        "fdtd_adjoint_transpose": ([P, C.c_int, C.POINTER(_dp)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


HEADER_SYMBOLS = [
    "fdtd_plan_create", "fdtd_plan_destroy", "fdtd_set_stream", "fdtd_sync",
    "fdtd_set_fields", "fdtd_get_fields", "fdtd_get_fields_f32", "fdtd_set_fields_f32",
    "fdtd_step", "fdtd_step_graph", "fdtd_step_static_scratch", "fdtd_get_step", "fdtd_step_timed", "fdtd_step_profile",
    "fdtd_get_probes", "fdtd_nfff_spectrum", "fdtd_nfff_ndata", "fdtd_nfff_series", "fdtd_get_map", "fdtd_get_nclasses",
    "fdtd_snapshot_size", "fdtd_snapshot_save", "fdtd_snapshot_restore",
    "fdtd_last_error", "fdtd_step_bytes",
    "fdtd_batch_create", "fdtd_batch_destroy", "fdtd_batch_size", "fdtd_batch_plan", "fdtd_batch_step",
    "fdtd_batch_step_graph", "fdtd_batch_sync", "fdtd_batch_tune", "fdtd_batch_config", "fdtd_batch_get_stream",
    "fdtd_set_design_eps", "fdtd_objective_value", "fdtd_adjoint_gradient", "fdtd_adjoint_transpose",
]


class FdtdError(RuntimeError):
    pass


def check(rc: int, what: str = "") -> None:
    if rc != OK:
        msg = load_library().fdtd_last_error().decode(errors="replace")
        raise FdtdError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")


def field_ptrs(arrs, ctype=C.c_double):
    arr_t = C.POINTER(ctype) * 6
    return arr_t(*[as_ptr(a, ctype) for a in arrs])
