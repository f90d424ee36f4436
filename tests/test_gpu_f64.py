"""FP64 reference-precision plans (FDTD_STORE_F64): fields, psi and ADE state
in FP64 and every update in FP64 on the general kernels.  Against the FP64
CPU oracle they agree to FP64 rounding (the GPU forms the Drude state in
difference form and contracts products into FMAs, so not bit for bit), far
below the FP32 path's 1e-5; and the FP32 path stays within 1e-5 of them."""
import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from gsvit_copy_b200.solver import Solver
from oracle.pyoracle import CpuSolver, series_spectrum
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu
TOL64 = 1e-10


def _f64(scene):
    scene.storage = abi.STORE_F64
    return scene


@pytest.mark.parametrize("kind", ["lintab", "ade", "pec", "full"])
def test_f64_random_state_matches_oracle(kind):
    s = _f64(plan.small_scene(kind, nsteps=120))
    g, o = Solver(s), CpuSolver(s)
    init = random_fields((s.xres, s.yres, s.zres), 11)
    g.set_fields(init)
    o.set_fields(init)
    g.step(120)
    o.step(120)
    errs = [rel_l2(a, b) for a, b in zip(g.fields(), o.fields())]
    assert max(errs) < TOL64, errs
    assert rel_l2(g.probes(), o.probes()) < TOL64


@pytest.mark.parametrize("kind", ["ade", "full"])
def test_f64_tsf_driven_farfield_matches_oracle(kind):
    s = _f64(plan.small_scene(kind, nsteps=200))
    g, o = Solver(s), CpuSolver(s)
    g.step(200)
    o.step(200)
    errs = [rel_l2(a, b) for a, b in zip(g.fields(), o.fields())]
    assert max(errs) < TOL64, errs
    assert rel_l2(g.probes(), o.probes()) < TOL64
    ref = series_spectrum(o.nfff_series(), s.nfff["omega"], s.dt)
    assert rel_l2(g.nfff_spectrum(), ref) < TOL64


def test_f64_snapshot_and_graph_bitwise():
    s = _f64(plan.small_scene("full", nsteps=64))
    a, b = Solver(s), Solver(s)
    init = random_fields((s.xres, s.yres, s.zres), 3)
    a.set_fields(init)
    b.set_fields(init)
    a.step(12)
    snap = a.snapshot()
    a.step(24)
    b.step(12)
    b.step_graph(24, chunk=8)
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)
    a.restore(snap)
    a.step(24)
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)


def test_f32_rough_surface_against_f64_run():
    """A 96^3 rough Drude-silver surface (the 512^3 workload's recipe, 16-cell
    CPML, TSF 30 deg, NFFF) from rest for 600 steps: the FP32 tiled run's
    probes, final E and far-field spectrum against the FP64 run."""
    s32 = plan.rough_surface_scene(res=96, nsteps=600, nfff_angles=(10, 19))
    s64 = _f64(plan.rough_surface_scene(res=96, nsteps=600, nfff_angles=(10, 19)))
    a, b = Solver(s32), Solver(s64)
    a.step(600)
    b.step(600)
    for x, y in zip(a.fields(abi.E_ALL), b.fields(abi.E_ALL)):
        if x is not None:
            assert rel_l2(x, y) < 1e-5
    assert rel_l2(a.probes(), b.probes()) < 1e-5
    assert rel_l2(a.nfff_spectrum(), b.nfff_spectrum()) < 1e-5
