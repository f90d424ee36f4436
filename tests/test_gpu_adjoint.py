"""The adjoint on the GPU (fdtd_adjoint_*): the design-region forward against
the FP64 oracle, the transposed step against the FP64 transpose of
oracle/adjoint.py, and the gradient against the FP64 adjoint gradient and
against finite differences of GPU runs.

Tolerances (relative L2): forward 1e-5 (at step 250, while the pulse is in
the box: later only a residual of ~3e-4 of the peak is left, where FP32
cancellation dominates); transposed step 1e-5 (FP32 against FP64); gradient
against the FP64 adjoint 1e-4; central finite differences of the FP32
objective 1e-3 of the largest derivative at h = 0.1 on eps_r (FP32 rounding
noise grows as 1/h: measured 1.8e-2 at h = 1e-3, 2.8e-3 at 1e-2, 4.7e-4 at
0.1; the FP64 check of tests/test_adjoint_oracle.py pins the discrete
adjoint to 1e-6 at h = 1e-4)."""
import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from gsvit_copy_b200.solver import Solver
from oracle import adjoint as A
from oracle.pyoracle import CpuSolver, series_spectrum
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu
NSTEPS = 600


def small_design_scene(nsteps=NSTEPS, seed=5, metal_cells=0):
    return plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=nsteps,
                              pulse_delay=2e-15, pulse_width=0.7e-15, seed=seed, metal_cells=metal_cells)


@pytest.mark.parametrize("tiles", ["0", "1"])
def test_design_forward_vs_oracle(tiles, monkeypatch):
    """tiles = 1: the design cells take the bulk tile layout's per-cell path."""
    monkeypatch.setenv("GSVIT_B200_TILES", tiles)
    s = small_design_scene(nsteps=250)
    obj = plan.cone_objective(s, nth=5, nph=7)
    g, o = Solver(s), CpuSolver(s.expanded())
    g.step(250)
    o.step(250)
    fg, fo = g.fields(), o.fields()
    for sl in (slice(0, 3), slice(3, 6)):   # E and H as vector fields (the x-polarised part is scattered light only)
        err = rel_l2(np.stack(fg[sl]), np.stack(fo[sl]))
        assert err < 1e-5, err
    spec = g.nfff_spectrum()
    ref = series_spectrum(o.nfff_series(), s.nfff["omega"], s.dt)
    assert rel_l2(spec, ref) < 1e-5, rel_l2(spec, ref)
    assert abs(g.objective_value(obj) / A.objective_value(o, obj) - 1) < 1e-5


@pytest.mark.parametrize("which", ["pec", "design", "ade", "full", "design_drude"])
def test_transposed_step_vs_fp64(which):
    """8 transposed steps from random (E, H) adjoints; the polarisation,
    E^{n-1} and psi adjoints start at zero on both sides ("ade" and "full"
    run the Drude / critical-point branch and the CPML inside it)."""
    if which in ("pec", "ade", "full"):
        s = plan.small_scene(which)
        s.tsf = None
    else:
        s = small_design_scene(nsteps=10, metal_cells=8 if which == "design_drude" else 0)
    g = Solver(s)
    L = A.LinearStep(CpuSolver(s.expanded()))
    rng = np.random.default_rng(4)
    shape = (s.xres, s.yres, s.zres)
    comps = [rng.standard_normal(shape) * (1.0 if c < 3 else 376.73) for c in range(6)]
    out = g.adjoint_transpose(comps, 8)
    ad = L.zero_state()
    for c in range(3):
        ad["E"][c][:] = comps[c]
        ad["H"][c][:] = comps[3 + c]
    for _ in range(8):
        L.adjoint(ad)
    ref = ad["E"] + ad["H"]
    errs = [rel_l2(a, b) for a, b in zip(out, ref)]
    assert max(errs) < 1e-5, errs


@pytest.mark.parametrize("metal", [0, 8])
def test_gradient_vs_fp64_adjoint(metal):
    """metal = 8: a Drude-silver layer across the bottom of the grid, inside
    the z0 CPML, so that the backward pass runs the transposed ADE branch."""
    s = small_design_scene(metal_cells=metal)
    obj = plan.cone_objective(s, nth=5, nph=7)
    g = Solver(s)
    J, grad = g.adjoint_gradient(obj, NSTEPS, checkpoint=128)
    J64, grad64 = A.gradient(s, obj, NSTEPS)
    print("J", J, J64, "grad rel", rel_l2(grad, grad64))
    assert abs(J / J64 - 1) < 1e-5
    assert rel_l2(grad, grad64) < 1e-4, rel_l2(grad, grad64)
    # the plan holds the forward state after the call
    assert g.step_count == NSTEPS
    assert abs(g.objective_value(obj) / J - 1) < 1e-12


def test_gradient_vs_finite_differences():
    s = plan.adjoint_scene(shape=(64, 64, 48), cpml_depth=8, design_shape=(16, 16, 4), glass_cells=6, nsteps=1200,
                           pulse_delay=4e-15, pulse_width=1.5e-15, seed=11)
    obj = plan.cone_objective(s, nth=7, nph=9)
    g = Solver(s)
    snap = g.snapshot()
    J, grad = g.adjoint_gradient(obj, 1200, checkpoint=200)
    rng = np.random.default_rng(3)
    cells = [tuple(int(rng.integers(0, n)) for n in grad.shape) for _ in range(8)]
    h = 0.1
    eps0 = s.design["eps"].copy()
    fd = []
    for q in cells:
        vals = []
        for sgn in (1, -1):
            e = eps0.copy()
            e[q] += sgn * h
            g.restore(snap)
            g.set_design_eps(e)
            g.step(1200)
            vals.append(g.objective_value(obj))
        fd.append((vals[0] - vals[1]) / (2 * h))
    g.set_design_eps(eps0)
    ad = np.array([grad[q] for q in cells])
    fd = np.array(fd)
    err = np.abs(ad - fd) / np.abs(grad).max()
    print("adjoint", ad, "fd", fd, "err", err)
    assert err.max() < 1e-3, err


def test_torch_autograd_wrapper():
    import torch
    from gsvit_copy_b200.adjoint import far_field_objective
    s = small_design_scene(nsteps=300)
    obj = plan.cone_objective(s, nth=5, nph=7)
    g = Solver(s)
    init = g.snapshot()
    eps = torch.tensor(s.design["eps"], dtype=torch.float64, requires_grad=True)
    J = far_field_objective(eps, g, obj, 300, 100, init)
    J.backward()
    g.restore(init)
    J2, grad = g.adjoint_gradient(obj, 300, 100)
    assert abs(J.item() / J2 - 1) < 1e-12
    # the objective's source is scattered with float atomics: the last bits vary between runs
    assert np.allclose(eps.grad.numpy(), grad, rtol=1e-5, atol=0)

