"""The library's host planner (gsvit_copy_b200/csrc/plan_host.cpp) on CPU.

The planner is plain C++; tests/host_plan_probe.cpp puts a C entry point over
it, and this file compiles both with g++ into pytest's temporary directory.
- The integer maps GSvit derives before its loop -- `bnds`
  (plan.c:5387-5416) and `sourceskip` (plan.c:5298-5326) -- equal the
  oracle's bit for bit.
- The per-cell coefficient classes index the planner's class table, and each
  cell's FP32 coefficients are the oracle's FP64 ones rounded to FP32: the H
  update da, db (yee.c:219-243), the ordinary E update ca, cb after get_cabs
  averaging (yee.c:1397-1493) where get_tbc keeps it, the dispersive-branch
  selection per component and the PEC zeroing rule (yee.c:1138-1237).
- The CPML grading of every face (becebhch, boundary.c:34-99) is the
  oracle's: b, c of E and H rounded to FP32, kappa exactly.
- The TSF auxiliary grid has the oracle's resolution (plan.c:1584-1595), and
  the dispersive variant is chosen exactly when an ADE material is used.
- An adjoint design region's per-cell E coefficients, at creation and after
  new permittivities, are the oracle's for the same scene with every design
  cell its own linear material (get_cabs averaging across the region's
  edges), rounded to FP32; the chain rule from dJ/dcb to dJ/d eps_r
  (design_gradient) agrees with central differences of those coefficients.
- The ADE coefficient sets restate GSvit's polarisation recursion
  (yee.c:923-1082) in difference form (Q = P_D^n - P_D^{n-1}, per pole
  p = P^n, q = P^n - P^{n-1}): driven alike, the two give the same E."""
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
    lib.host_plan_classes.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.c_size_t]
    lib.host_plan_classes.restype = C.c_int
    fp, dp = C.POINTER(C.c_float), C.POINTER(C.c_double)
    lib.host_plan_cpml.argtypes = [C.c_void_p, C.c_int] + [fp] * 4 + [dp] * 2 + [C.c_int]
    lib.host_plan_cpml.restype = C.c_int
    lib.host_plan_scalars.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
    lib.host_plan_scalars.restype = C.c_int
    lib.host_plan_design.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_size_t]
    lib.host_plan_design.restype = C.c_longlong
    lib.host_plan_design_gradient.argtypes = [C.c_void_p] + [C.c_void_p] * 3
    lib.host_plan_design_gradient.restype = C.c_int
    lib.host_plan_ades.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.host_plan_ades.restype = C.c_int
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


# DevClass (gsvit_copy_b200/csrc/fdtd_internal.h), 64 bytes
DEV_CLASS = np.dtype([("ca", "<f4", 3), ("flags", "<u4"), ("cb", "<f4", 3), ("tsfe", "<f4"), ("da", "<f4"),
                      ("db", "<f4"), ("ade", "<i4"), ("pad0", "<f4"), ("cba", "<f4", 3), ("pad1", "<f4")])
CF_ADE_BRANCH, CF_PEC_SHIFT = 0x8, 4


@pytest.mark.parametrize("name", list(SCENES))
def test_planner_coefficients_are_the_oracle_rounded_to_fp32(probe, name):
    from oracle import adjoint as A
    assert DEV_CLASS.itemsize == 64
    s = SCENES[name]()
    cls, ncls = _map(probe, s, abi.MAP_CLASS)
    desc, keep = s.desc()
    table = np.zeros(256, dtype=DEV_CLASS)
    err = C.create_string_buffer(512)
    assert probe.host_plan_classes(C.addressof(desc), table.ctypes.data, 256, err, len(err)) == ncls
    per_cell = table[:ncls][cls.ravel()]
    o = CpuSolver(s)
    n = cls.size
    ca, cb, da, db = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n), np.zeros(n)
    fl = np.zeros(n, dtype=np.int32)
    assert A._lib().oracle_get_coeffs(o.h, A._p(ca), A._p(cb), A._p(da), A._p(db), fl.ctypes.data_as(A._ip)) == 0
    o.close()
    f32 = lambda x: x.astype(np.float32)
    assert np.array_equal(per_cell["da"], f32(da)) and np.array_equal(per_cell["db"], f32(db))
    flags = per_cell["flags"]
    branch = (fl & 64) != 0                             # the cell takes the dispersive branch
    assert np.array_equal((flags & CF_ADE_BRANCH) != 0, branch)
    for a in range(3):
        ordinary = ((fl >> a) & 1) == 1                 # get_tbc keeps the ordinary update of component a
        assert np.array_equal(per_cell["ca"][:, a][ordinary], f32(ca[a * n:(a + 1) * n])[ordinary])
        assert np.array_equal(per_cell["cb"][:, a][ordinary], f32(cb[a * n:(a + 1) * n])[ordinary])
        assert np.array_equal(((flags >> a) & 1) == 1, ~ordinary & branch)
        assert np.array_equal(((flags >> (CF_PEC_SHIFT + a)) & 1) == 1, ((fl >> (3 + a)) & 1) == 1)


@pytest.mark.parametrize("name", ["full", "rough64", "sphere60"])
def test_planner_cpml_grading_is_the_oracle(probe, name):
    from oracle import adjoint as A
    s = SCENES[name]()
    desc, keep = s.desc()
    o = CpuSolver(s)
    fp, dp = C.POINTER(C.c_float), C.POINTER(C.c_double)
    for face in range(6):
        mine = [np.zeros(64, np.float32) for _ in range(4)] + [np.zeros(64) for _ in range(2)]
        n = probe.host_plan_cpml(C.addressof(desc), face, *[a.ctypes.data_as(fp) for a in mine[:4]],
                                 *[a.ctypes.data_as(dp) for a in mine[4:]], 64)
        ref = [np.zeros(64) for _ in range(6)]
        m = A._lib().oracle_get_cpml(o.h, face, *[A._p(a) for a in ref])
        assert n == m and n > 0, (face, n, m)
        for q in range(4):                               # be, ce, bh, ch
            assert np.array_equal(mine[q][:n], ref[q][:m].astype(np.float32)), (face, q)
        for q in (4, 5):                                 # kappa_e, kappa_h
            assert np.array_equal(mine[q][:n], ref[q][:m]), (face, q)
    o.close()


@pytest.mark.parametrize("name", list(SCENES))
def test_planner_aux_grid_and_variant(probe, name):
    s = SCENES[name]()
    desc, keep = s.desc()
    jres, has_ade, maxpoles = C.c_int(), C.c_int(), C.c_int()
    assert probe.host_plan_scalars(C.addressof(desc), C.byref(jres), C.byref(has_ade), C.byref(maxpoles)) == 0
    o = CpuSolver(s)
    aux_res = o._f("aux_res")
    aux_res.argtypes = [C.c_void_p]
    aux_res.restype = C.c_int
    assert jres.value == (aux_res(o.h) if s.tsf else 0)
    o.close()
    used = np.unique(s.mat) if s.mat is not None else np.array([0])
    uses_ade = any(s.mats[int(i)].type == abi.MAT_ADE for i in used)
    assert has_ade.value == int(uses_ade)
    assert maxpoles.value in (0, 2)


def _oracle_coeffs(scene):
    from oracle import adjoint as A
    o = CpuSolver(scene)
    n = scene.ncells
    ca, cb, da, db = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n), np.zeros(n)
    fl = np.zeros(n, dtype=np.int32)
    assert A._lib().oracle_get_coeffs(o.h, A._p(ca), A._p(cb), A._p(da), A._p(db), fl.ctypes.data_as(A._ip)) == 0
    o.close()
    shape = (3, scene.xres, scene.yres, scene.zres)
    return ca.reshape(shape), cb.reshape(shape)


def test_planner_design_coefficients_are_the_oracle(probe):
    s = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=10,
                           pulse_delay=2e-15, pulse_width=0.7e-15, seed=5)
    new_eps = np.random.default_rng(9).uniform(1.5, 4.0, s.design["eps"].shape)
    for eps in (None, new_eps):
        desc, keep = s.desc()
        abox = (C.c_int * 6)()
        buf = np.zeros(6 * 4096, np.float32)
        arg = None if eps is None else np.ascontiguousarray(eps, dtype=np.float64).ctypes.data
        n = probe.host_plan_design(C.addressof(desc), arg, abox, buf.ctypes.data, buf.size)
        assert n > 0
        mine = buf[:6 * n].reshape(-1, 6)
        ref_scene = s
        if eps is not None:
            ref_scene = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3,
                                           nsteps=10, pulse_delay=2e-15, pulse_width=0.7e-15, seed=5)
            ref_scene.design["eps"] = eps.copy()
        ca, cb = _oracle_coeffs(ref_scene.expanded())
        b = list(abox)
        box = (slice(b[0], b[1]), slice(b[2], b[3]), slice(b[4], b[5]))
        assert n == (b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4])
        for a in range(3):
            assert np.array_equal(mine[:, a], ca[a][box].ravel().astype(np.float32)), ("ca", a)
            assert np.array_equal(mine[:, 3 + a], cb[a][box].ravel().astype(np.float32)), ("cb", a)


def test_planner_design_gradient_vs_central_differences(probe):
    """J(eps) = sum w * cb(eps) over the affected cells: design_gradient(w) must
    be dJ/d eps_r.  cb is FP32, so h = 1e-2 on eps_r in [1.5, 4] leaves a
    rounding noise near 1e-5 and a truncation error near 1e-5 of the largest
    derivative."""
    s = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=10,
                           pulse_delay=2e-15, pulse_width=0.7e-15, seed=5)
    rng = np.random.default_rng(21)
    eps = np.ascontiguousarray(rng.uniform(1.5, 4.0, s.design["eps"].shape))
    desc, keep = s.desc()
    abox = (C.c_int * 6)()
    buf = np.zeros(6 * 4096, np.float32)

    def cb_of(e):
        n = probe.host_plan_design(C.addressof(desc), np.ascontiguousarray(e).ctypes.data, abox, buf.ctypes.data,
                                   buf.size)
        assert n > 0
        return buf[:6 * n].reshape(-1, 6)[:, 3:].astype(np.float64)

    w = rng.standard_normal(cb_of(eps).shape)
    w = np.ascontiguousarray(w / np.abs(cb_of(eps)).max())
    grad = np.zeros(eps.size)
    assert probe.host_plan_design_gradient(C.addressof(desc), eps.ctypes.data, w.ctypes.data, grad.ctypes.data) == 0
    h = 1e-2
    fd = np.zeros(eps.size)
    flat = eps.ravel()
    for q in range(eps.size):
        up, dn = flat.copy(), flat.copy()
        up[q] += h
        dn[q] -= h
        fd[q] = ((w * cb_of(up.reshape(eps.shape))).sum() - (w * cb_of(dn.reshape(eps.shape))).sum()) / (2 * h)
    err = np.abs(grad - fd).max() / np.abs(fd).max()
    print("design gradient vs central differences:", err)
    assert err < 1e-3, err


# DevAde (gsvit_copy_b200/csrc/fdtd_internal.h)
DEV_ADE = np.dtype([("c0dx", "<f4"), ("c2", "<f4"), ("c3", "<f4"), ("qe", "<f4"), ("ma0", "<f4"), ("a2", "<f4"),
                    ("pe", "<f4", 2), ("qpe", "<f4", 2), ("rp", "<f4", 2), ("rq", "<f4", 2), ("bp2", "<f4", 2),
                    ("bp3", "<f4", 2), ("bp4", "<f4", 2)])


def _reference_ade(m, dx, curl):
    """GSvit's update of one dispersive component, FP64 (yee.c:923-929 for E,
    yee.c:1070-1082 for P_D and the critical-point P, then the n-1 copies)."""
    e = ep = 0.0
    dp = dpp = 0.0
    p, pp = [0.0, 0.0], [0.0, 0.0]
    out = np.empty(len(curl))
    for n, cu in enumerate(curl):
        e1 = (m.ade_c0 * cu / dx + m.ade_c1 * (-m.ade_a0 * dpp + (1 - m.ade_a1) * dp)
              + sum(m.ade_c1 * (-m.ade_bp0[q] * pp[q] + (1 - m.ade_bp1[q]) * p[q]) for q in range(2))
              + m.ade_c2 * ep + m.ade_c3 * e)
        dpn = m.ade_a0 * dpp + m.ade_a1 * dp + m.ade_a2 * (ep + 2 * e + e1)
        pn = [m.ade_bp0[q] * pp[q] + m.ade_bp1[q] * p[q] + m.ade_bp2[q] * ep + m.ade_bp3[q] * e + m.ade_bp4[q] * e1
              for q in range(2)]
        dpp, dp, pp, p, ep, e = dp, dpn, p, pn, e, e1
        out[n] = e1
    return out


def _difference_ade(a, curl):
    """The difference form the kernels run, in FP64 arithmetic with the given coefficients."""
    e = ep = 0.0
    qd = 0.0
    p, q = [0.0, 0.0], [0.0, 0.0]
    out = np.empty(len(curl))
    for n, cu in enumerate(curl):
        v = (a["c0dx"] * cu + a["qe"] * qd + sum(a["qpe"][k] * q[k] + a["pe"][k] * p[k] for k in range(2))
             + a["c2"] * ep + a["c3"] * e)
        qd = a["ma0"] * qd + a["a2"] * (ep + 2 * e + v)
        for k in range(2):
            qn = a["rp"][k] * p[k] + a["rq"][k] * q[k] + a["bp2"][k] * ep + a["bp3"][k] * e + a["bp4"][k] * v
            q[k] = qn
            p[k] += qn
        ep, e = e, v
        out[n] = v
    return out


def _exact_sets(m, dx):
    """The planner's formulas (plan_host.cpp) without the rounding to FP32."""
    return {"c0dx": m.ade_c0 / dx, "c2": m.ade_c2, "c3": m.ade_c3, "qe": m.ade_c1 * m.ade_a0, "ma0": -m.ade_a0,
            "a2": m.ade_a2, "pe": [m.ade_c1 * ((1.0 - m.ade_bp0[k]) - m.ade_bp1[k]) for k in range(2)],
            "qpe": [m.ade_c1 * m.ade_bp0[k] for k in range(2)],
            "rp": [(m.ade_bp0[k] + m.ade_bp1[k]) - 1.0 for k in range(2)], "rq": [-m.ade_bp0[k] for k in range(2)],
            "bp2": list(m.ade_bp2), "bp3": list(m.ade_bp3), "bp4": list(m.ade_bp4)}


@pytest.mark.parametrize("name", ["ade", "full", "rough64", "rough64_lorentz"])
def test_planner_ade_sets_restate_the_recursion(probe, name):
    s = (plan.rough_surface_scene(res=64, nsteps=10, nfff_angles=None, material="lorentz")
         if name == "rough64_lorentz" else SCENES[name]())
    desc, keep = s.desc()
    sets = np.zeros(16, dtype=DEV_ADE)
    record = C.c_int()
    n = probe.host_plan_ades(C.addressof(desc), sets.ctypes.data, 16, C.byref(record))
    assert record.value == DEV_ADE.itemsize
    ade_mats = [m for m in s.mats[1:] if m.type == abi.MAT_ADE]
    assert n == len(ade_mats) > 0
    rng = np.random.default_rng(17)
    for a, m in zip(sets[:n], ade_mats):
        curl = rng.standard_normal(2000) * s.dx / m.ade_c0          # c0 * curl / dx of order 1
        ref = _reference_ade(m, s.dx, curl)
        exact = _difference_ade(_exact_sets(m, s.dx), curl)
        fp32 = _difference_ade(a, curl)
        scale = np.linalg.norm(ref)
        assert np.linalg.norm(exact - ref) / scale < 1e-12    # the algebra of the restatement
        assert np.linalg.norm(fp32 - ref) / scale < 1e-5      # with the coefficients the kernels get
