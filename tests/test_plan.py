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


def test_batch_scenes_follow_the_batched_workload():
    """48 seeded instances: x, y in {64, 96, 128, 192}, z in {64, 96, 128},
    8-cell CPML on every face, incidence 0-60 deg from +z, rms height 5-20 nm
    (1-4 cells of 5 nm), Drude silver or the single-pole Lorentz substrate,
    both present; the same seed gives the same instances."""
    sc, again = plan.batch_scenes(48, nsteps=64), plan.batch_scenes(48, nsteps=64)
    assert len(sc) == 48
    kinds = set()
    for s, t in zip(sc, again):
        assert s.xres in (64, 96, 128, 192) and s.yres in (64, 96, 128, 192) and s.zres in (64, 96, 128)
        assert all(s.cpml[f][0] == 8 for f in range(6))
        assert 120.0 <= math.degrees(s.tsf["theta"]) <= 180.0
        assert 1.0 - 1e-9 <= float(np.std(s.meta["height_map"])) <= 4.0 + 1e-9
        m = s.mats[1]
        if m.drude_omega_p > 0:
            kinds.add("drude")
            assert m.drude_omega_p == plan.f32(1.38e16) and m.drude_nu == plan.f32(2.73e13)
        else:
            kinds.add("lorentz")
            a, _, big_omega, gamma = plan.lorentz_as_cp(5.0, 2.0, 4e15, 1e14)
            assert m.cp_omega[0] == plan.f32(big_omega) and m.cp_gamma[0] == plan.f32(gamma)
            assert m.cp_a[0] == plan.f32(a) and m.cp_a[1] == 0.0
        assert (s.xres, s.yres, s.zres) == (t.xres, t.yres, t.zres)
        assert np.array_equal(s.mat, t.mat)
    assert kinds == {"drude", "lorentz"}


def test_cone_objective_weights_cover_the_cone():
    """The appended far points lie within the cone (10 deg about theta = 20
    deg, up to the integer rounding of a point 640 cells out), the objective
    indexes exactly them, istart covers every point, and the weights
    sin(theta) dtheta dphi sum to the cone's solid angle 2 pi (1 - cos 10 deg)
    within the quadrature error of the grid."""
    for nth, nph, tol in ((9, 13, 0.02), (41, 61, 0.01)):
        s = plan.rough_surface_scene(res=64, nsteps=10, nfff_angles=(4, 7))
        n0 = len(s.nfff["points"])
        obj = plan.cone_objective(s, nth=nth, nph=nph)
        assert np.array_equal(obj["points"], np.arange(n0, len(s.nfff["points"])))
        assert len(s.nfff["istart"]) == len(s.nfff["points"])
        d = s.nfff["points"][obj["points"]] - np.array([32, 32, 32])
        d = d / np.linalg.norm(d, axis=1)[:, None]
        axis = np.array([math.sin(math.radians(20)), 0.0, math.cos(math.radians(20))])
        assert np.degrees(np.arccos(np.clip(d @ axis, -1, 1))).max() < 10.05
        cone = 2 * math.pi * (1 - math.cos(math.radians(10)))
        assert abs(obj["weights"].sum() / cone - 1) < tol
