"""Generate the golden fixtures of tests/golden/ (run in a checkout that has
GSvit's sources, so that oracle/_ref/libgsvit_ref.so can be built).

    python tests/golden/make_golden.py [--selftests] [--small]

selftest_<id>.npz   far-field time series of GSvit's own self-tests
                    (make_test, tests.c:93-268) for the TSF + CPML + NFFF ids
                    31111 (electric voxel box, 200^3) and 35011 (PEC box, 100^3
                    and 200^3), computed by the FP64 oracle and checked here against
                    the reference's golden files tests/selftests/<res><id> with
                    the tests.c comparison (relative L2 of |F| per row); the
                    agreement is stored in the fixture as `pin_rel_l2`.
ref_small_<kind>.npz  GSvit's own CPU stepping code (compiled from its sources
                    into oracle/_ref) on the small mixed scenes of
                    gsvit_copy_b200.plan.small_scene, TSF-driven for 120 steps:
                    the bnds / sourceskip maps, the probe series, the far-field
                    series, and the six field components at 512 seeded cells.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gsvit_copy_b200 import abi, plan  # noqa: E402
from oracle import pyoracle  # noqa: E402

SELFTEST_DIR = os.path.join(os.environ.get("GSVIT_REF", "/root/reference"), "tests", "selftests")
# 10031111 is left out: its golden file predates the current far-field buffer
# length (50000 rows instead of 2702) and GSvit's own stepping code, compiled
# from its sources (oracle/_ref), misses it by 0.8 % under the tests.c metric,
# while it reproduces 10035011, 20031111 and 20035011 to ~1e-6.
SELFTESTS = [(100, "35011"), (200, "31111"), (200, "35011")]
SMALL_KINDS = ["lintab", "ade", "pec", "full"]
SMALL_STEPS = 120
NSAMPLE = 512


def selftest_rel(series, golden):
    """tests.c metric: relative L2 of the per-row magnitude |F| (the reference's
    files store -F, the sign of its output convention, which |F| ignores)."""
    mine = series.T
    vg = np.sqrt((golden[:, 1:] ** 2).sum(1))
    vm = np.sqrt((mine ** 2).sum(1))
    n = min(len(vg), len(vm))
    return float(np.sqrt(((vg[:n] - vm[:n]) ** 2).sum() / (vm[:n] ** 2).sum()))


def selftest_fixture(res, code):
    nsteps = 2 * res + 1
    s = plan.selftest_scene(code, res, nsteps)
    o = pyoracle.CpuSolver(s, "oracle")
    o.step(nsteps)
    series = o.nfff_series()[0]
    istart = o.nfff_istart()
    golden = np.loadtxt(os.path.join(SELFTEST_DIR, f"{res}{code}"))
    rel = selftest_rel(series, golden)
    n = min(len(golden), series.shape[1])
    comp = [float(np.linalg.norm(golden[:n, 1 + c] + series[c, :n]) / np.linalg.norm(golden[:n, 1 + c]))
            for c in range(3)]
    print(f"selftest {res}{code}: |F| rel L2 {rel:.2e}, components {['%.2e' % x for x in comp]}")
    assert rel < 1e-5 and max(comp) < 1e-5
    np.savez_compressed(os.path.join(HERE, f"selftest_{res}{code}.npz"), series=series, istart=istart,
                        nsteps=nsteps, pin_rel_l2=rel, pin_comp_rel_l2=np.array(comp))


def sample_cells(shape, n=NSAMPLE, seed=7):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, s, n) for s in shape], axis=1).astype(np.int32)


def small_fixture(kind):
    s = plan.small_scene(kind, nsteps=SMALL_STEPS)
    r = pyoracle.CpuSolver(s, "reference")
    r.step(SMALL_STEPS)
    f = r.fields()
    cells = sample_cells(f[0].shape)
    vals = np.stack([c[cells[:, 0], cells[:, 1], cells[:, 2]] for c in f], axis=1)
    np.savez_compressed(os.path.join(HERE, f"ref_small_{kind}.npz"),
                        bnds=r.map(abi.MAP_BNDS).astype(np.int8), sourceskip=r.map(abi.MAP_SOURCESKIP).astype(np.int8),
                        probes=r.probes(), nfff_series=r.nfff_series(), cells=cells, values=vals,
                        norms=np.array([np.linalg.norm(c) for c in f]), nsteps=SMALL_STEPS)
    print(f"ref_small_{kind}: norms {[float('%.4g' % np.linalg.norm(c)) for c in f]}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--selftests", action="store_true")
    ap.add_argument("--small", action="store_true")
    a = ap.parse_args()
    both = not (a.selftests or a.small)
    if a.small or both:
        if not pyoracle.reference_available():
            raise SystemExit("oracle/_ref/libgsvit_ref.so is missing: run `make -C oracle ref` first")
        for k in SMALL_KINDS:
            small_fixture(k)
    if a.selftests or both:
        for res, code in SELFTESTS:
            selftest_fixture(res, code)


if __name__ == "__main__":
    main()
