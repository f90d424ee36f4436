"""16-bit field storage (FDTD_STORE_F16 / FDTD_STORE_BF16): fields and CPML
psi slabs are held as FP16 or BF16 in HBM, with H and psi scaled by powers
of two; every update computes in FP32.  BF16 stores round stochastically
(round to nearest stalls sub-ulp increments: far-field error 0.28 at 128^3).

Tolerances (relative L2 against the FP64 oracle, 40 steps from a seeded
white-noise state, the worst case for rounding): FP16 5e-3, BF16 4e-2.
Far field of the rough-surface workload at 128^3 from rest (the physical
pulse, 4000 steps, the 91 x 181 far grid) against an FP64 run of the same
scene: FP32 within 1e-5, FP16 within the 1e-3 storage target; BF16 misses
that target (expected failure, reason in the test)."""
import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from gsvit_copy_b200.solver import Batch, Solver
from oracle.pyoracle import CpuSolver
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu

FIELD_TOL = {abi.STORE_F16: 5e-3, abi.STORE_BF16: 4e-2}
STORES = [pytest.param(abi.STORE_F16, id="f16"), pytest.param(abi.STORE_BF16, id="bf16")]
# k rows of 64 cells are 128 bytes at 16 bits: the TMA tiles run, and the
# interior box is large enough for the bulk layout
SHAPE = (40, 48, 64)


def _scene(kind, storage, nsteps=40):
    s = plan.small_scene(kind, shape=SHAPE, nsteps=nsteps)
    s.storage = storage
    return s


@pytest.mark.parametrize("storage", STORES)
@pytest.mark.parametrize("kind", ["full", "ade", "lintab"])
def test_fields_vs_oracle(kind, storage):
    s = _scene(kind, storage)
    g, o = Solver(s), CpuSolver(s)
    init = random_fields((s.xres, s.yres, s.zres), 5)
    g.set_fields(init)
    o.set_fields(init)
    g.step(40)
    o.step(40)
    errs = [rel_l2(a, b) for a, b in zip(g.fields(), o.fields())]
    print(kind, storage, "field errors", ["%.2e" % e for e in errs])
    assert max(errs) < FIELD_TOL[storage], errs
    prof = g.step_profile(1)
    assert prof["bulk_bytes"] > 0, "the TMA bulk kernel did not take the interior"


@pytest.mark.parametrize("storage", STORES)
def test_set_get_round_trip_is_exact_for_representable_values(storage):
    """Values representable in the storage type (H after the 2^9 scale) come
    back bit-exact; the host conversion rounds to nearest even."""
    s = _scene("lintab", storage)
    g = Solver(s)
    rng = np.random.default_rng(3)
    shape = (s.xres, s.yres, s.zres)
    # small integers times powers of two are exact in FP16 and BF16 alike
    comps = [rng.integers(-64, 65, size=shape).astype(np.float64) * 2.0 ** -6 * (1.0 if c < 3 else 2.0 ** -9)
             for c in range(6)]
    g.set_fields(comps)
    back = g.fields()
    for a, b in zip(back, comps):
        assert np.array_equal(a, b)


@pytest.fixture(scope="module")
def f64_rough_128():
    """The rough Drude-silver surface at 128^3 (the 512^3 workload's recipe:
    16-cell CPML, TSF 30 deg, 91 x 181 far grid) lit from rest by the TSF
    pulse (peak at step 2392), 4000 steps, in FP64 storage and arithmetic."""
    s = plan.rough_surface_scene(res=128, nsteps=4000)
    s.storage = abi.STORE_F64
    g = Solver(s)
    g.step_graph(4000)
    out = {"spec": g.nfff_spectrum(), "probes": g.probes(), "E": g.fields(abi.E_ALL)[:3]}
    g.close()
    return out


BF16_FAR = ("BF16 misses the 1e-3 far-field target: 1.4e-3 against the FP64 run at 512^3 (8 significant "
            "bits with stochastic rounding)")


@pytest.mark.parametrize("storage", [pytest.param(abi.STORE_F32, id="f32"), pytest.param(abi.STORE_F16, id="f16"),
                                     pytest.param(abi.STORE_BF16, id="bf16",
                                                  marks=pytest.mark.xfail(reason=BF16_FAR, strict=False))])
def test_far_field_rough_surface_128_vs_f64(storage, f64_rough_128):
    """The same run with FP32, FP16 and BF16 storage against the FP64 run:
    far-field spectrum within 1e-5 (FP32) and 1e-3 (16-bit, the storage
    target); the probe series and final E are printed."""
    s = plan.rough_surface_scene(res=128, nsteps=4000)
    s.storage = storage
    g = Solver(s)
    g.step_graph(4000)
    spec, probes, E = g.nfff_spectrum(), g.probes(), g.fields(abi.E_ALL)[:3]
    g.close()
    ref = f64_rough_128
    err = rel_l2(spec, ref["spec"])
    print("storage", storage, "far field %.3e" % err, "probes %.3e" % rel_l2(probes, ref["probes"]),
          "E", ["%.2e" % rel_l2(x, y) for x, y in zip(E, ref["E"])])
    assert np.abs(ref["spec"]).max() > 0
    assert err < (1e-5 if storage == abi.STORE_F32 else 1e-3), err


@pytest.mark.parametrize("storage", STORES)
def test_batch_matches_one_by_one(storage):
    """A batch of 16-bit instances gives the bits of each instance stepped alone."""
    scenes = []
    for kind in ("full", "lintab"):
        scenes.append(_scene(kind, storage, nsteps=20))
    alone = []
    for s in scenes:
        g = Solver(s)
        g.step(20)
        alone.append(g.fields())
        g.close()
    b = Batch(scenes)
    b.step(20)
    for q in range(len(scenes)):
        for x, y in zip(b[q].fields(), alone[q]):
            assert np.array_equal(x, y)


def test_batch_rejects_mixed_storage():
    a, b = _scene("lintab", abi.STORE_F16), _scene("lintab", abi.STORE_F32)
    with pytest.raises(RuntimeError, match="storage"):
        Batch([a, b])
