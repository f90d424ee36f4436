"""The TMA tile kernels over the whole grid (interior box plus the CPML tiles
of the x/y and z layouts) against the FP64 CPU oracle, through the C ABI.

Scenes are large enough for all three tile layouts, with CPML depths 6, 8, 12
(kappa_max 2, CFS alpha), Drude / critical-point metal inside the z0 slab
(the ADE-in-CPML branch), PEC, tabulated dielectrics, a TSF box and an NFFF
box outside the slabs, and random initial fields so that every cell is active.
Tolerance: relative L2 1e-5 for FP32 fields and probes against FP64."""
import numpy as np
import pytest

from gsvit_copy_b200 import plan
from gsvit_copy_b200.solver import Solver
from oracle.pyoracle import CpuSolver, series_spectrum
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(autouse=True)
def _tiles_on(monkeypatch):
    """These CPML depths (6-12) take the slab kernels by default; force the tiles."""
    monkeypatch.setenv("GSVIT_B200_TILES", "1")


def tiled_scene(kind, shape, depth, nsteps):
    s = plan.small_scene(kind, shape=shape, nsteps=nsteps)
    xr, yr, zr = shape
    s.cpml = plan.cpml_all(depth, 3, -1, 2.0, 0.02, s.dx)
    m = depth + 3
    s.tsf["box"] = ((m, m, m), (xr - m, yr - m, zr - m))
    s.nfff["box"] = ((m - 1, m - 1, m - 1), (xr - m + 1, yr - m + 1, zr - m + 1))
    return s


CASES = [("full", (40, 52, 72), 8), ("ade", (36, 48, 64), 6), ("full", (44, 64, 96), 12), ("lintab", (33, 47, 68), 8)]


@pytest.mark.parametrize("kind,shape,depth", CASES)
def test_tiles_random_state_parity(kind, shape, depth):
    s = tiled_scene(kind, shape, depth, 60)
    g, o = Solver(s), CpuSolver(s)
    init = random_fields(shape, 21)
    g.set_fields(init)
    o.set_fields(init)
    g.step(60)
    o.step(60)
    errs = [rel_l2(a, b) for a, b in zip(g.fields(), o.fields())]
    assert max(errs) < TOL, errs
    assert rel_l2(g.probes(), o.probes()) < TOL


@pytest.mark.parametrize("kind,shape,depth", CASES[:2])
def test_tiles_tsf_driven_farfield(kind, shape, depth):
    s = tiled_scene(kind, shape, depth, 160)
    g, o = Solver(s), CpuSolver(s)
    g.step(160)
    o.step(160)
    errs = [rel_l2(a, b) for a, b in zip(g.fields(), o.fields())]
    assert max(errs) < TOL, errs
    assert rel_l2(g.probes(), o.probes()) < TOL
    ref = series_spectrum(o.nfff_series(), s.nfff["omega"], s.dt)
    assert rel_l2(g.nfff_spectrum(), ref) < TOL


def test_tiles_use_three_layouts_and_match_slab_path(monkeypatch):
    """The same run through the tiles and through the slab kernels (the path of
    plans without tiles, selected by GSVIT_B200_NO_BULK) agree to FP32
    rounding; the tiled step launches the bulk and the three CPML kinds."""
    s = tiled_scene("full", (40, 52, 72), 8, 40)
    init = random_fields((s.xres, s.yres, s.zres), 4)
    g = Solver(s)
    g.set_fields(init)
    prof = g.step_profile(1)
    # aux grid, TSF faces, four tile kinds (bulk; CPML x, y and z slabs), NFFF sampling and ring fold
    assert int(prof["launches_per_step"]) == 8, prof
    g.step(29)
    monkeypatch.setenv("GSVIT_B200_NO_BULK", "1")
    h = Solver(s)
    monkeypatch.delenv("GSVIT_B200_NO_BULK")
    h.set_fields(init)
    h.step(30)
    for a, b in zip(g.fields(dtype=np.float32), h.fields(dtype=np.float32)):
        assert rel_l2(a, b) < 2e-6
