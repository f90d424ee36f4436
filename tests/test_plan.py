"""Host-side planner (gsvit_copy_b200.plan): the planning rules GSvit applies
before its stepping loop, checked on CPU."""
import math

import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from oracle import pyoracle
from oracle.pyoracle import CpuSolver
from tests._util import random_fields


def test_dt_is_courant_fraction():
    dx = 5e-9
    dt = plan.plan_dt(dx, dx, dx, 0.5)
    assert math.isclose(dt * plan.C0 * math.sqrt(3) / dx, 0.5, rel_tol=1e-14)


def test_sigma_opt():
    assert math.isclose(plan.cpml_sigma_opt(3, 10e-9), 0.8 * 3 / (377 * 10e-9), rel_tol=1e-15)


def test_sphere_map_matches_cell_centre_float_test():
    """is_in_sphere(i+0.5f, j+0.5f, k+0.5f) in float arithmetic, small grid, plain loops."""
    shape = (13, 11, 12)
    mat = np.zeros(shape, dtype=np.int32)
    c = (6.3, 5.1, 5.9)
    r = 3.7
    plan.sphere_map(mat, c, r, 2)
    f = np.float32
    ref = np.zeros(shape, dtype=np.int32)
    for i in range(shape[0]):
        for j in range(shape[1]):
            for k in range(shape[2]):
                x, y, z = f(i) + f(0.5), f(j) + f(0.5), f(k) + f(0.5)
                d = (x - f(c[0])) * (x - f(c[0])) + (y - f(c[1])) * (y - f(c[1]))
                d = d + (z - f(c[2])) * (z - f(c[2]))
                if d <= f(r) * f(r):
                    ref[i, j, k] = 2
    assert np.array_equal(mat, ref)
    assert mat.sum() > 0


def test_height_map_statistics_and_seed():
    h = plan.gaussian_height_map(128, 96, 2.0, 10.0, seed=5)
    assert abs(h.mean()) < 1e-12
    assert math.isclose(h.std(), 2.0, rel_tol=1e-12)
    assert np.array_equal(h, plan.gaussian_height_map(128, 96, 2.0, 10.0, seed=5))
    assert not np.array_equal(h, plan.gaussian_height_map(128, 96, 2.0, 10.0, seed=6))
    # correlated: neighbouring heights are close compared with the rms
    assert np.abs(np.diff(h, axis=0)).mean() < 0.5 * h.std()


def test_spherical_area_and_istart():
    pts = plan.spherical_area(91, 181, 5120, 0.0, 0.0, plan.G_PI / 2, 2 * plan.G_PI, 512, 512, 512)
    assert pts.shape == (91 * 181, 3)
    assert tuple(pts[0]) == (256, 256, 256 + 5120)
    ist = plan.nfff_istart(pts, plan.plan_dt(5e-9, 5e-9, 5e-9, 0.5), 5e-9, shared=True)
    assert (ist == ist[0]).all() and ist[0] > 0


def test_tsf_pulse_is_g_quantised():
    w = plan.tsf_pulse(200, 20e-6, 10, plan.plan_dt(1e-6, 1e-6, 1e-6, 1.0), 5.0)
    assert all(float("%g" % v) == v for v in w)
    assert np.abs(w).max() > 0


def test_rough_surface_scene_geometry():
    s = plan.rough_surface_scene(res=96, nsteps=10, nfff_angles=(5, 9))
    h = s.meta["height_map"]
    z0 = s.meta["surface_z"]
    k = np.arange(s.zres)[None, None, :] + 0.5
    assert np.array_equal(s.mat, (k < (z0 + h)[:, :, None]).astype(np.int32))
    (ti, tj, tk), (tI, tJ, tK) = s.tsf["box"]
    (ni, nj, nk), (nI, nJ, nK) = s.nfff["box"]
    d = s.cpml[0][0]
    assert d < ni < ti and tI < nI < s.xres - d
    assert s.tsf["skip"][abi.FACE_Z0] == 1
    assert len(s.nfff["points"]) == 45
    assert ((s.probes >= 0) & (s.probes < [s.xres, s.yres, s.zres])).all()


@pytest.mark.skipif(not pyoracle.reference_available(), reason="oracle/_ref not built")
def test_electric_voxel_mode_oracle_vs_reference():
    """MATMODE ELECTRIC (per-voxel epsilon / sigma arrays, no material table)."""
    s = plan.small_scene("lintab", nsteps=30)
    rng = np.random.default_rng(4)
    s.matmode = abi.MATMODE_ELECTRIC
    s.mats = []
    s.mat = None
    shape = (s.xres, s.yres, s.zres)
    s.epsilon = np.full(shape, np.float32(plan.EPS0), dtype=np.float32)
    s.sigma = np.zeros(shape, dtype=np.float32)
    plan.voxel_box(s.epsilon, (8, 5, 6), (18, 15, 20), np.float32(plan.f32(2.0) * plan.EPS0))
    plan.voxel_box(s.sigma, (10, 6, 8), (14, 12, 12), np.float32(50.0))
    s.epsilon *= (1 + 0.1 * rng.random(shape)).astype(np.float32)
    o, r = CpuSolver(s, "oracle"), CpuSolver(s, "reference")
    init = random_fields(shape, 9)
    o.set_fields(init)
    r.set_fields(init)
    o.step(30)
    r.step(30)
    for w in (abi.MAP_BNDS, abi.MAP_SOURCESKIP):
        assert np.array_equal(o.map(w), r.map(w))
    for a, b in zip(o.fields(), r.fields()):
        assert np.array_equal(a, b)
