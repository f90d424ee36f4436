"""Batches (fdtd_batch_*): many uneven instances stepped in lockstep, one
launch per kernel for all of them, against the same scenes stepped one by one
(bit-identical: the same per-cell arithmetic) and, for the Lorentz substrate
that only the batch workload uses, against the FP64 oracle (relative L2 1e-5)."""
import numpy as np
import pytest

from gsvit_copy_b200 import plan
from gsvit_copy_b200.solver import Batch, Solver
from oracle.pyoracle import CpuSolver, series_spectrum
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu


def _scenes(nsteps):
    sc = [plan.rough_surface_scene(res=64, yres=48, zres=64, nsteps=nsteps, cpml_depth=8, tsf_margin=6, seed=3,
                                   material="lorentz", theta_deg=160.0, nfff_angles=(4, 7)),
          plan.rough_surface_scene(res=40, yres=72, zres=48, nsteps=nsteps, cpml_depth=8, tsf_margin=6, seed=4,
                                   nfff_angles=(4, 7)),
          plan.small_scene("full", nsteps=nsteps),
          plan.small_scene("lintab", shape=(26, 22, 30), nsteps=nsteps)]   # zres % 4 != 0: slab kernels only
    return sc


def _init(views, scenes):
    """Seeded random fields everywhere (the TSF pulse enters only after ~2500 steps)."""
    for q, (v, sc) in enumerate(zip(views, scenes)):
        v.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 100 + q))


def _compare(a, b):
    for x, y in zip(a.fields(dtype=np.float32), b.fields(dtype=np.float32)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.probes(), b.probes())


def test_batch_matches_one_by_one_bitwise():
    n = 90
    scenes = _scenes(n)
    batch = Batch(scenes)
    _init(batch.views, scenes)
    batch.step(40)
    batch.step_graph(50, chunk=10)
    batch.sync()
    for q, sc in enumerate(scenes):
        alone = Solver(sc)
        alone.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 100 + q))
        alone.step(n)
        _compare(batch[q], alone)
        if sc.nfff is not None and len(sc.nfff.get("omega", [])):
            assert np.array_equal(batch[q].nfff_spectrum(), alone.nfff_spectrum())
        assert batch[q].step_count == n
        alone.close()
    batch.close()


def test_batch_tune_keeps_state_and_results():
    n = 30
    scenes = _scenes(n)
    batch = Batch(scenes)
    _init(batch.views, scenes)
    batch.step(10)
    report = batch.tune(trial_steps=2)
    assert len(report) == 10 and all(r[2] > 0 for r in report)
    cfg = batch.config()
    # the bulk work list holds only the instances without TMA tiles (here the
    # one whose zres is not a multiple of 4)
    assert cfg["items"] >= 0 and cfg["planes_per_item"] in (0, 8, 16, 32, 64)
    batch.step(20)
    batch.sync()
    for q, sc in enumerate(scenes):
        alone = Solver(sc)
        alone.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 100 + q))
        alone.step(n)
        _compare(batch[q], alone)
        alone.close()
    batch.close()


def test_batch_lorentz_instance_vs_oracle():
    n = 160
    scenes = _scenes(n)
    batch = Batch(scenes)
    _init(batch.views, scenes)
    batch.step(n)
    o = CpuSolver(scenes[0])
    o.set_fields(random_fields((scenes[0].xres, scenes[0].yres, scenes[0].zres), 100))
    o.step(n)
    for a, b in zip(batch[0].fields(), o.fields()):
        assert rel_l2(a, b) < 1e-5
    assert rel_l2(batch[0].probes(), o.probes()) < 1e-5
    ref = series_spectrum(o.nfff_series(), scenes[0].nfff["omega"], scenes[0].dt)
    assert rel_l2(batch[0].nfff_spectrum(), ref) < 1e-5
    batch.close()
