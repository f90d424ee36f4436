"""The library's host planner (gsvit_copy_b200/csrc/plan_host.cpp) on CPU.

The planner is plain C++; tests/host_plan_probe.cpp puts a C entry point over
it, and this file compiles both with g++ into pytest's temporary directory.
The integer maps GSvit derives before its loop -- `bnds` (plan.c:5387-5416)
and `sourceskip` (plan.c:5298-5326) -- must equal the oracle's bit for bit;
the per-cell coefficient classes must index the planner's class table."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from oracle.pyoracle import CpuSolver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INCLUDE = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "vector_types.h")):
        pytest.skip("needs g++ and the CUDA headers")
    out = str(tmp_path_factory.mktemp("hostplan") / "libhostplan.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-I", CUDA_INCLUDE,
                           os.path.join(ROOT, "tests", "host_plan_probe.cpp"),
                           os.path.join(ROOT, "gsvit_copy_b200", "csrc", "plan_host.cpp"), "-o", out])
    lib = C.CDLL(out)
    lib.host_plan_map.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.c_char_p,
                                  C.c_size_t]
    lib.host_plan_map.restype = C.c_int
    return lib


def _map(lib, scene, which):
    desc, keep = scene.desc()
    out = np.empty((scene.xres, scene.yres, scene.zres), dtype=np.int32)
    ncls = C.c_int(0)
    err = C.create_string_buffer(512)
    rc = lib.host_plan_map(C.addressof(desc), which, out.ctypes.data, out.size, C.byref(ncls), err, len(err))
    assert rc == 0, err.value.decode()
    return out, ncls.value


SCENES = {
    "lintab": lambda: plan.small_scene("lintab"),
    "ade": lambda: plan.small_scene("ade"),
    "pec": lambda: plan.small_scene("pec"),
    "full": lambda: plan.small_scene("full"),
    "rough64": lambda: plan.rough_surface_scene(res=64, nsteps=10, nfff_angles=None),
    "sphere60": lambda: plan.sphere_scene(res=60, nsteps=10, radius=12.0),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_planner_maps_bit_exact_vs_oracle(probe, name):
    s = SCENES[name]()
    o = CpuSolver(s)
    for w in (abi.MAP_BNDS, abi.MAP_SOURCESKIP):
        m, _ = _map(probe, s, w)
        assert np.array_equal(m, o.map(w)), (name, w)
    o.close()


@pytest.mark.parametrize("name", ["full", "rough64"])
def test_planner_classes_index_the_table(probe, name):
    s = SCENES[name]()
    cls, ncls = _map(probe, s, abi.MAP_CLASS)
    assert 1 <= ncls <= 256
    assert cls.min() >= 0 and cls.max() < ncls
    assert len(np.unique(cls)) == ncls      # every class of the table is used by some cell
