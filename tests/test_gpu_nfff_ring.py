"""The running DFT buffers E samples for 8 steps before it folds them into the
FP64 accumulators.  Reading the spectrum in the middle of a block folds the
pending steps early; snapshots carry the unfolded samples.  Neither may change
what the accumulators hold afterwards: a run read at 13 steps and again at 45
gives the spectrum of the same run read only at 45, and a snapshot taken at
13 steps and restored replays the same spectrum (bit for bit: the same
products are added in the same order; an early fold leaves zeros in the
slots it used, and adding a zero leaves a sum unchanged)."""
import numpy as np
import pytest

from gsvit_copy_b200 import plan
from gsvit_copy_b200.solver import Batch, Solver
from oracle.pyoracle import CpuSolver, series_spectrum
from tests._util import rel_l2, random_fields

pytestmark = pytest.mark.gpu


def _scene():
    return plan.small_scene("full", nsteps=64)


def _solver(sc):
    g = Solver(sc)
    g.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 41))
    return g


def test_mid_block_read_leaves_the_spectrum_unchanged():
    sc = _scene()
    a, b = _solver(sc), _solver(sc)
    a.step(13)
    early = a.nfff_spectrum()           # 5 samples of the second block folded early
    assert np.isfinite(early).all() and np.abs(early).max() > 0
    a.step(3)
    a.nfff_spectrum()                   # a read right at a block boundary folds nothing
    a.step(29)
    b.step(45)
    assert np.array_equal(a.nfff_spectrum(), b.nfff_spectrum())
    a.close()
    b.close()


def test_mid_block_snapshot_replays():
    sc = _scene()
    g = _solver(sc)
    g.step(13)
    snap = g.snapshot()
    g.step(30)
    first = g.nfff_spectrum()
    g.restore(snap)
    g.step(30)
    assert np.array_equal(g.nfff_spectrum(), first)
    g.close()


def test_ring_spectrum_vs_oracle_off_block():
    """43 steps (not a multiple of 8) against the FP64 oracle's DFT of its series."""
    sc = _scene()
    g = _solver(sc)
    o = CpuSolver(sc)
    o.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 41))
    g.step(43)
    o.step(43)
    ref = series_spectrum(o.nfff_series(), sc.nfff["omega"], sc.dt)
    assert rel_l2(g.nfff_spectrum(), ref) < 1e-5
    g.close()


def test_batch_with_an_instance_without_running_dft():
    """A batch may mix plans with and without a running DFT: the DFT kernel
    leaves the plain instance alone, and each instance matches its own run."""
    with_dft, plain = _scene(), plan.small_scene("ade", nsteps=64)
    plain.nfff = None
    scenes = [with_dft, plain]
    batch = Batch(scenes)
    for q, (v, sc) in enumerate(zip(batch.views, scenes)):
        v.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 50 + q))
    batch.step(21)
    batch.sync()
    for q, sc in enumerate(scenes):
        alone = Solver(sc)
        alone.set_fields(random_fields((sc.xres, sc.yres, sc.zres), 50 + q))
        alone.step(21)
        for x, y in zip(batch[q].fields(dtype=np.float32), alone.fields(dtype=np.float32)):
            assert np.array_equal(x, y)
        if sc.nfff is not None:
            assert np.array_equal(batch[q].nfff_spectrum(), alone.nfff_spectrum())
        alone.close()
    batch.close()
