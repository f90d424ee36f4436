"""The FP64 adjoint restatement (oracle/adjoint.py) pinned on the CPU: its
forward step against the C oracle (bit-exact), its transpose by the
dot-product identity <M^n x, y> = <x, (M^T)^n y>, and its gradient of the
far-field objective against central finite differences of the oracle's own
objective (FP64, h = 1e-4 on eps_r) -- also with Drude / critical-point
materials, whose dispersive branch (yee.c:914-1108, with the CPML inside it)
the restatement steps and transposes."""
import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from oracle import adjoint as A
from oracle.pyoracle import CpuSolver
from tests._util import random_fields


def _dot(a, b):
    d = sum(float(np.sum(a[k][c] * b[k][c])) for k in ("E", "H") for c in range(3))
    for k in ("ep", "dp", "dpp"):
        if k in a:
            d += sum(float(np.sum(a[k][c] * b[k][c])) for c in range(3))
    for k in ("p", "pp"):
        if k in a:
            d += sum(float(np.sum(a[k][c][q] * b[k][c][q])) for c in range(3) for q in range(2))
    return d


def _randomise_ade(L, st, rng, scale):
    """Random dispersive state on the cells of the dispersive branch (elsewhere
    it is not part of the step's state)."""
    for k in ("ep", "dp", "dpp"):
        for c in range(3):
            st[k][c][:] = np.where(L.ade, rng.standard_normal(L.shape) * scale, 0.0)
    for k in ("p", "pp"):
        for c in range(3):
            for q in range(2):
                st[k][c][q][:] = np.where(L.ade, rng.standard_normal(L.shape) * scale, 0.0)


def _copy(st):
    out = {k: [v.copy() for v in st[k]] for k in ("E", "H")}
    for k in ("ep", "dp", "dpp"):
        if k in st:
            out[k] = [v.copy() for v in st[k]]
    for k in ("p", "pp"):
        if k in st:
            out[k] = [[v.copy() for v in w] for w in st[k]]
    return out


@pytest.mark.parametrize("kind", ["lintab", "pec", "ade", "full"])
def test_forward_restatement_is_the_oracle_step(kind):
    s = plan.small_scene(kind)
    s.tsf = None
    o = CpuSolver(s)
    L = A.LinearStep(o)
    init = random_fields((s.xres, s.yres, s.zres), 3)
    o.set_fields(init)
    st = L.zero_state()
    for a in range(3):
        st["E"][a][:] = init[a]
        st["H"][a][:] = init[3 + a]
    o.step(5)
    for _ in range(5):
        L.forward(st)
    for a, b in zip(st["E"] + st["H"], o.fields()):
        assert np.array_equal(a, b)
    assert all(np.abs(p).max() > 0 for f in st["pe"] for p in st["pe"][f])


@pytest.mark.parametrize("kind", ["pec", "design", "ade", "full", "design_drude"])
def test_transpose_dot_product(kind):
    if kind in ("pec", "ade", "full"):
        s = plan.small_scene(kind)
        s.tsf = None
    else:
        s = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=10,
                               metal_cells=4 if kind == "design_drude" else 0).expanded()
    L = A.LinearStep(CpuSolver(s))
    assert L.has_ade == (kind in ("ade", "full", "design_drude"))
    rng = np.random.default_rng(1)
    x, y = L.zero_state(), L.zero_state()
    for a in range(3):
        x["E"][a][:] = rng.standard_normal(L.shape)
        x["H"][a][:] = rng.standard_normal(L.shape) / 377
        y["E"][a][:] = rng.standard_normal(L.shape)
        y["H"][a][:] = rng.standard_normal(L.shape) * 377
    if L.has_ade:
        _randomise_ade(L, x, rng, 1e-11)
        _randomise_ade(L, y, rng, 1e11)
    x0, y0 = _copy(x), _copy(y)
    for _ in range(6):
        L.forward(x)
        L.adjoint(y)
    lhs, rhs = _dot(x, y0), _dot(x0, y)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_gradient_vs_finite_differences_fp64():
    n = 600
    s = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=n,
                           pulse_delay=2e-15, pulse_width=0.7e-15)
    obj = plan.cone_objective(s, nth=5, nph=7)
    J, g = A.gradient(s, obj, n)
    assert J > 0
    cells = [(0, 0, 0), (1, 2, 1), (3, 3, 0), (2, 1, 1)]
    fd = A.objective_fd(s, obj, n, cells, 1e-4)
    ad = np.array([g[q] for q in cells])
    assert np.max(np.abs(ad - fd) / np.abs(fd)) < 1e-6, (ad, fd)


def test_gradient_vs_finite_differences_fp64_drude():
    """The same with a Drude-silver layer under the glass (inside the z0 CPML
    and across the x and y slabs): the adjoint sweep runs through the ADE
    branch and the CPML inside it."""
    n = 600
    s = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=n,
                           pulse_delay=2e-15, pulse_width=0.7e-15, metal_cells=8)
    obj = plan.cone_objective(s, nth=5, nph=7)
    J, g = A.gradient(s, obj, n)
    assert J > 0
    cells = [(0, 0, 0), (1, 2, 1), (3, 3, 0)]
    fd = A.objective_fd(s, obj, n, cells, 1e-4)
    ad = np.array([g[q] for q in cells])
    assert np.max(np.abs(ad - fd) / np.abs(fd)) < 1e-6, (ad, fd)


def test_design_descriptor_validation():
    import ctypes as C
    s = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=10)
    lib = abi.load_library()
    for box, text in [((2, 6, 14, 18, 17, 19), "CPML"), ((14, 18, 14, 18, 20, 23), "TSF box")]:
        s2 = plan.adjoint_scene(shape=(32, 32, 32), cpml_depth=6, design_shape=(4, 4, 2), glass_cells=3, nsteps=10)
        i0, i1, j0, j1, k0, k1 = box
        s2.design = dict(box=box, eps=np.full((i1 - i0, j1 - j0, k1 - k0), 2.0))
        d, keep = s2.desc()
        h = C.c_void_p()
        rc = lib.fdtd_plan_create(C.byref(d), 0, C.byref(h))
        assert rc == -1, rc   # FDTD_E_INVALID
        assert text in lib.fdtd_last_error().decode()
