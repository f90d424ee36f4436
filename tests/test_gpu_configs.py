"""The measured workloads on the GPU against the FP64 oracle (and, through the
committed fixtures, against GSvit's own self-test golden files).

Tolerance: relative L2 1e-5 for FP32 fields, probe series and far-field
spectra against the FP64 CPU path."""
import os

import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from gsvit_copy_b200.solver import Solver
from oracle.pyoracle import CpuSolver, series_spectrum
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu
TOL = 1e-5
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_sphere_100_full_run():
    """Dielectric sphere, 100^3, 10-cell CPML, TSF box inset 15, 1000 steps:
    Ex/Ez probe series and the final E field."""
    s = plan.sphere_scene(res=100, nsteps=1000)
    g, o = Solver(s), CpuSolver(s)
    g.step(1000)
    o.step(1000)
    fg, fo = g.fields(abi.E_ALL), o.fields()
    for c in range(3):
        assert rel_l2(fg[c], fo[c]) < TOL, (c, rel_l2(fg[c], fo[c]))
    pg, po = g.probes(), o.probes()
    for c in (0, 2):
        assert rel_l2(pg[:, :, c], po[:, :, c]) < TOL
    assert np.abs(po[:, :, 0]).max() > 0.01   # rising edge of the 15 fs-delayed pulse (1000 steps = 9.6 fs)


@pytest.mark.parametrize("name", ["20031111", "20035011"])
def test_selftest_farfield_series_vs_reference_golden(name):
    """GSvit self-tests 31111 (electric voxel box) and 35011 (PEC box) at
    200^3, 401 steps, DT_MULT 1: the exact time-domain far-field series of the
    GPU run against the fixture pinned to the reference's golden file."""
    g0 = np.load(os.path.join(GOLD, f"selftest_{name}.npz"))
    res, code = int(name[:3]), name[3:]
    s = plan.selftest_scene(code, res, int(g0["nsteps"]))
    s.nfff["series"] = True
    g = Solver(s)
    g.step(int(g0["nsteps"]))
    ser = g.nfff_series()[0]
    ref = g0["series"]
    assert ser.shape == ref.shape
    assert rel_l2(ser, ref) < TOL, rel_l2(ser, ref)
    assert np.abs(ref).max() > 0


@pytest.mark.parametrize("name", ["20035011"])
def test_selftest_farfield_spectrum_at_courant_limit(name):
    """The running-DFT spectrum at DT_MULT 1, where a few dozen (cell, point)
    pairs have a step-dependent retarded index in the reference: agreement
    with the DFT of the golden series is bounded by those pairs (< 2e-3)."""
    g0 = np.load(os.path.join(GOLD, f"selftest_{name}.npz"))
    res, code = int(name[:3]), name[3:]
    s = plan.selftest_scene(code, res, int(g0["nsteps"]))
    w0 = 2 * plan.G_PI * plan.C0 / 20e-6
    s.nfff["omega"] = np.array([0.5 * w0, w0, 1.5 * w0])
    g = Solver(s)
    g.step(int(g0["nsteps"]))
    err = rel_l2(g.nfff_spectrum(), series_spectrum(g0["series"][None], s.nfff["omega"], s.dt))
    assert err < 2e-3, err


def test_rough_surface_128_reduced():
    """The rough Drude-silver workload at 128^3 (16-cell CPML, TSF 30 deg with
    the k0 face skipped, NFFF at 3 wavelengths, 10 x 19 far grid), started
    from a seeded random state so that every region is active, 150 steps."""
    s = plan.rough_surface_scene(res=128, nsteps=150, nfff_angles=(10, 19))
    g, o = Solver(s), CpuSolver(s)
    init = random_fields((s.xres, s.yres, s.zres), 17)
    g.set_fields(init)
    o.set_fields(init)
    g.step(150)
    o.step(150)
    for a, b in zip(g.fields(), o.fields()):
        assert rel_l2(a, b) < TOL
    assert rel_l2(g.probes(), o.probes()) < TOL
    spec = g.nfff_spectrum()
    ref = series_spectrum(o.nfff_series(), s.nfff["omega"], s.dt)
    assert rel_l2(spec, ref) < TOL, rel_l2(spec, ref)
    for w in (abi.MAP_BNDS, abi.MAP_SOURCESKIP):
        assert np.array_equal(g.map(w), o.map(w))


@pytest.mark.slow
def test_rough_surface_512_full_size_random_state():
    """The full 512^3 workload for 4 steps from a seeded random state: bulk
    tiles, all six CPML slabs, the ADE silver and the TSF faces at full size."""
    s = plan.rough_surface_scene(res=512, nsteps=8, nfff_angles=None)
    g, o = Solver(s), CpuSolver(s)
    rng = np.random.default_rng(5)
    init = [rng.standard_normal(g.shape).astype(np.float32) * (1.0 if c < 3 else 1 / 376.73) for c in range(6)]
    g.set_fields(init)
    o.set_fields(init)
    del init
    for w in (abi.MAP_BNDS, abi.MAP_SOURCESKIP):
        assert np.array_equal(g.map(w), o.map(w))
    g.step(4)
    o.step(4)
    fo = o.fields()
    o.close()
    fg = g.fields(dtype=np.float32)
    for a, b in zip(fg, fo):
        assert rel_l2(a, b) < TOL
