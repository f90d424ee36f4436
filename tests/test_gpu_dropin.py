"""The drop-in for GSvit's src3d/gpu.c (gsvit_copy_b200/dropin/gpu_b200.c):
GSvit's own planned structures stepped through its GPU branch (svit.c:240-256,
sv_pool_gpu_*) on the B200 library, against the same structures stepped
through its CPU branch.  Fields, point outputs and the far-field series land in
GSvit's own host structures (mp->d, outpointdata, rpoints) and must agree
within relative L2 1e-5."""
import numpy as np
import pytest

from gsvit_copy_b200 import plan
from tests import _dropin
from tests._util import rel_l2, random_fields

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not _dropin.available(), reason="oracle/_ref/libgsvit_dropin.so not built")]
TOL = 1e-5


@pytest.mark.parametrize("kind", ["lintab", "ade", "full"])
def test_dropin_gpu_branch_matches_cpu_branch(kind):
    s = plan.small_scene(kind, nsteps=160)
    cpu, gpu = _dropin.DropinRun(s, gpu=False), _dropin.DropinRun(s, gpu=True)
    init = random_fields((s.xres, s.yres, s.zres), 5)
    cpu.set_fields(init)
    gpu.set_fields(init)
    cpu.step(160)
    gpu.step(100)
    gpu.step(60)
    gpu.finish()
    for a, b in zip(gpu.fields(), cpu.fields()):
        assert rel_l2(a, b) < TOL
    assert rel_l2(gpu.probes(), cpu.probes()) < TOL
    sg, sc = gpu.nfff_series(), cpu.nfff_series()
    assert np.abs(sc).max() > 0
    assert rel_l2(sg, sc) < TOL
