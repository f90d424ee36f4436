"""The FP64 CPU oracle pinned against GSvit itself.

1. against GSvit's own CPU stepping code compiled from its sources
   (oracle/_ref/libgsvit_ref.so; skipped where it was not built),
2. against the committed fixtures of tests/golden/ that the reference produced
   (ref_small_*) or that were checked against the reference's own self-test
   golden files (selftest_*),
3. against those golden files themselves where GSvit's tree is present.
"""
import os

import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from oracle import pyoracle
from oracle.pyoracle import CpuSolver
from tests._util import rel_l2, random_fields

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KINDS = ["lintab", "ade", "pec", "full"]
needs_ref = pytest.mark.skipif(not pyoracle.reference_available(), reason="oracle/_ref not built")


def _load(name):
    return np.load(os.path.join(GOLD, name))


@needs_ref
@pytest.mark.parametrize("kind", KINDS)
def test_oracle_bit_exact_vs_reference_random_state(kind):
    """Every code path active from step 0 (CPML, ADE, PEC, TSF, domain edges)."""
    s = plan.small_scene(kind, nsteps=40)
    o, r = CpuSolver(s, "oracle"), CpuSolver(s, "reference")
    init = random_fields((s.xres, s.yres, s.zres), 3)
    o.set_fields(init)
    r.set_fields(init)
    o.step(40)
    r.step(40)
    for w in (abi.MAP_BNDS, abi.MAP_SOURCESKIP, abi.MAP_MAT):
        assert np.array_equal(o.map(w), r.map(w))
    for a, b in zip(o.fields(), r.fields()):
        assert np.array_equal(a, b)
    assert np.array_equal(o.probes(), r.probes())


@needs_ref
@pytest.mark.parametrize("kind", ["lintab", "full"])
def test_oracle_bit_exact_vs_reference_tsf_nfff(kind):
    s = plan.small_scene(kind, nsteps=150)
    o, r = CpuSolver(s, "oracle"), CpuSolver(s, "reference")
    o.step(150)
    r.step(150)
    for a, b in zip(o.fields(), r.fields()):
        assert np.array_equal(a, b)
    assert np.array_equal(o.nfff_istart(), r.nfff_istart())
    assert np.array_equal(o.nfff_series(), r.nfff_series())
    ea, ha = o.aux()
    eb, hb = r.aux()
    assert np.array_equal(ea, eb) and np.array_equal(ha, hb)


@pytest.mark.parametrize("kind", KINDS)
def test_oracle_vs_reference_fixture(kind):
    g = _load(f"ref_small_{kind}.npz")
    n = int(g["nsteps"])
    s = plan.small_scene(kind, nsteps=n)
    o = CpuSolver(s, "oracle")
    assert np.array_equal(o.map(abi.MAP_BNDS), g["bnds"].astype(np.int32))
    assert np.array_equal(o.map(abi.MAP_SOURCESKIP), g["sourceskip"].astype(np.int32))
    o.step(n)
    f = o.fields()
    cells = g["cells"]
    vals = np.stack([c[cells[:, 0], cells[:, 1], cells[:, 2]] for c in f], axis=1)
    assert rel_l2(vals, g["values"]) < 1e-12
    assert np.allclose([np.linalg.norm(c) for c in f], g["norms"], rtol=1e-12, atol=0)
    assert rel_l2(o.probes(), g["probes"]) < 1e-12
    assert rel_l2(o.nfff_series(), g["nfff_series"]) < 1e-12


SELFTEST_DIR = os.path.join(os.environ.get("GSVIT_REF", "/root/reference"), "tests", "selftests")


@pytest.mark.parametrize("code", ["35011"])
def test_oracle_vs_selftest_fixture(code):
    """GSvit self-test make_test id 35011 at 100^3 (201 steps)."""
    g = _load(f"selftest_100{code}.npz")
    s = plan.selftest_scene(code, 100, int(g["nsteps"]))
    o = CpuSolver(s, "oracle")
    o.step(int(g["nsteps"]))
    assert np.array_equal(o.nfff_istart(), g["istart"])
    assert rel_l2(o.nfff_series()[0], g["series"]) < 1e-12
    assert float(g["pin_rel_l2"]) < 1e-5


@pytest.mark.skipif(not os.path.isdir(SELFTEST_DIR), reason="GSvit's self-test golden files are not present")
@pytest.mark.parametrize("name", ["10035011", "20031111", "20035011"])
def test_selftest_fixture_matches_reference_golden_file(name):
    """tests.c comparison (relative L2 of |F| per output row) of the committed
    fixture against the reference's own golden file; the files hold -F."""
    g = _load(f"selftest_{name}.npz")
    ref = np.loadtxt(os.path.join(SELFTEST_DIR, name))
    ser = g["series"]
    n = min(ref.shape[0], ser.shape[1])
    vg = np.sqrt((ref[:n, 1:] ** 2).sum(1))
    vm = np.sqrt((ser[:, :n] ** 2).sum(0))
    assert np.sqrt(((vg - vm) ** 2).sum() / (vm ** 2).sum()) < 1e-5
    for c in range(3):
        assert rel_l2(-ser[c, :n], ref[:n, 1 + c]) < 1e-5
