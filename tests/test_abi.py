"""The C ABI library: it loads on a machine without a GPU, exports every entry
point include/gsvit_b200.h declares, its ctypes mirror matches the C layout,
and descriptor validation errors come back as status codes (no GPU work)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gsvit_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdtd_\w+)\s*\(", text)))


def test_library_loads_and_exports_header_symbols():
    lib = abi.load_library()
    declared = header_functions()
    assert declared, "no declarations parsed"
    assert sorted(abi.HEADER_SYMBOLS) == declared
    out = subprocess.run(["nm", "-D", "--defined-only", abi.lib_path()], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (fdtd_\w+)", out))
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        assert getattr(lib, s) is not None


def test_library_is_sm100a():
    """The library carries sm_100a device code (checked through the ELF section list only)."""
    out = subprocess.run(["readelf", "-S", abi.lib_path()], capture_output=True, text=True, check=True).stdout
    assert ".nv_fatbin" in out


LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include "gsvit_b200.h"
#define P(T, F) printf(#T "." #F " %zu\n", offsetof(T, F))
int main(void) {
    printf("fdtd_material %zu\nfdtd_cpml_face %zu\nfdtd_tsf %zu\nfdtd_nfff %zu\nfdtd_desc %zu\n",
           sizeof(fdtd_material), sizeof(fdtd_cpml_face), sizeof(fdtd_tsf), sizeof(fdtd_nfff), sizeof(fdtd_desc));
    P(fdtd_material, ade_c3); P(fdtd_tsf, wave); P(fdtd_tsf, skipdepth); P(fdtd_nfff, omega);
    P(fdtd_nfff, skip_hi); P(fdtd_desc, mats); P(fdtd_desc, cpml); P(fdtd_desc, tsf); P(fdtd_desc, nfff);
    P(fdtd_desc, probes); P(fdtd_desc, storage);
    return 0;
}
"""


def test_ctypes_mirror_matches_c_layout(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                              check=True).stdout.strip().splitlines())
    assert int(got["fdtd_material"]) == C.sizeof(abi.Material)
    assert int(got["fdtd_cpml_face"]) == C.sizeof(abi.CpmlFace)
    assert int(got["fdtd_tsf"]) == C.sizeof(abi.Tsf)
    assert int(got["fdtd_nfff"]) == C.sizeof(abi.Nfff)
    assert int(got["fdtd_desc"]) == C.sizeof(abi.Desc)
    assert int(got["fdtd_material.ade_c3"]) == abi.Material.ade_c3.offset
    assert int(got["fdtd_tsf.wave"]) == abi.Tsf.wave.offset
    assert int(got["fdtd_tsf.skipdepth"]) == abi.Tsf.skipdepth.offset
    assert int(got["fdtd_nfff.omega"]) == abi.Nfff.omega.offset
    assert int(got["fdtd_nfff.skip_hi"]) == abi.Nfff.skip_hi.offset
    for f in ("mats", "cpml", "tsf", "nfff", "probes", "storage"):
        assert int(got[f"fdtd_desc.{f}"]) == getattr(abi.Desc, f).offset, f


def _create(desc):
    lib = abi.load_library()
    h = C.c_void_p()
    rc = lib.fdtd_plan_create(C.byref(desc), 0, C.byref(h))
    return rc, lib.fdtd_last_error().decode()


@pytest.mark.parametrize("mutate,code,text", [
    (lambda s, d: setattr(d, "abi_version", 99), -1, "ABI version"),
    (lambda s, d: setattr(d, "xres", 2), -1, "at least 3"),
    (lambda s, d: setattr(d, "dt", -1.0), -1, "positive"),
    (lambda s, d: setattr(d, "dy", d.dx * 2), -2, "non-cubic"),
    (lambda s, d: setattr(d, "storage", 7), -1, "storage"),
    (lambda s, d: setattr(d.tsf, "theta", 4.0), -1, "theta"),
    (lambda s, d: setattr(d.cpml[0], "depth", 1), -1, "CPML depth"),
])
def test_descriptor_validation_without_gpu(mutate, code, text):
    s = plan.small_scene("full")
    d, keep = s.desc()
    mutate(s, d)
    rc, msg = _create(d)
    assert rc == code, (rc, msg)
    assert text.lower() in msg.lower(), msg


def test_material_index_out_of_range():
    s = plan.small_scene("lintab")
    s.mat = s.mat.copy()
    s.mat[3, 4, 5] = len(s.mats)
    d, keep = s.desc()
    rc, msg = _create(d)
    assert rc == -1
    assert "out of range" in msg


def test_probe_outside_grid():
    s = plan.small_scene("lintab")
    s.probes = np.asarray([(s.xres, 0, 0)], dtype=np.int32)
    d, keep = s.desc()
    rc, msg = _create(d)
    assert rc == -1 and "probe" in msg


def test_null_arguments():
    lib = abi.load_library()
    assert lib.fdtd_plan_create(None, 0, None) == -1
    assert lib.fdtd_step(None, 1) == -1
    assert lib.fdtd_sync(None) == -1
    assert lib.fdtd_plan_destroy(None) == 0


DROPIN_SO = os.path.join(ROOT, "oracle", "_ref", "libgsvit_dropin.so")
GSVIT_GPU_FAMILY = ["sv_gpu_new", "sv_pool_gpu_init", "sv_pool_gpu_apply_source_hstep", "sv_pool_gpu_apply_source_estep",
                    "sv_pool_gpu_ystep_h", "sv_pool_gpu_ystep_e", "sv_pool_gpu_copyto", "sv_pool_gpu_copyfrom",
                    "sv_pool_gpu_getsum", "sv_pool_gpu_boundary_copy", "sv_pool_gpu_boundary_hstep",
                    "sv_pool_gpu_boundary_estep", "sv_pool_gpu_apply_farfield", "sv_pool_gpu_getpoints",
                    "sv_pool_gpu_getforce", "sv_pool_gpu_apply_pfarfield"]


@pytest.mark.skipif(not os.path.exists(DROPIN_SO), reason="drop-in test build not present")
def test_dropin_exports_gsvit_gpu_family():
    """The drop-in for src3d/gpu.c defines sv_gpu_new and every sv_pool_gpu_*
    function GSvit's loop calls (pool.h:98-128) and links libgsvit_b200."""
    out = subprocess.run(["nm", "-D", "--defined-only", DROPIN_SO], capture_output=True, text=True, check=True).stdout
    defined = set(re.findall(r"\bT (sv_\w+)", out))
    assert not [s for s in GSVIT_GPU_FAMILY if s not in defined]
    deps = subprocess.run(["readelf", "-d", DROPIN_SO], capture_output=True, text=True, check=True).stdout
    assert "libgsvit_b200.so" in deps


@pytest.mark.skipif(not os.path.exists(DROPIN_SO), reason="drop-in test build not present")
def test_dropin_build_cpu_branch_is_gsvit():
    """Compiled with UCUDA (SvPool then carries its gpu member), GSvit's CPU
    branch in the drop-in build still gives the bits of the plain build."""
    from oracle.pyoracle import CpuSolver
    from tests import _dropin
    s = plan.small_scene("full", nsteps=20)
    a, b = _dropin.DropinRun(s, gpu=False), CpuSolver(s, "reference")
    a.step(20)
    b.step(20)
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)
