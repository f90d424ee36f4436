"""GSvit's own CUDA path -- src3d/gpu.c and gpu_kernels.cu compiled unmodified
for sm_100a into oracle/_ref/libgsvit_refcuda.so and stepped through the GPU
branch of svit.c:240-256 -- is the measured context baseline of bench.py's
reference arm.  Here it is checked against the FP64 oracle on the small
scene's CPML (kappa 2, a 0.02), TSF plane wave, NFFF box and probes in
vacuum, from rest, so that the time it reports is the time of the same
update.  Its arithmetic is FP32 with -use_fast_math (configure.ac:57); the
tolerance, relative L2 per field component after 60 steps, is 2e-4.

GSvit's GPU branch is not its CPU branch everywhere, so the check stays in
vacuum: its E kernels take a cell's own epsilon and sigma where the CPU
branch averages them over the interface (gpu_kernels.cu eKernel_tab against
yee.c get_cabs), and its ADE cells inside the CPML take the ADE update
without kappa and the psi_E correction with the per-cell (vacuum)
coefficient (gpu_kernels.cu eKernel_cpml_tab, cpmleKernelx) where the CPU
branch has its ADE-in-CPML update (yee.c:950-1057): a rough Drude surface
that reaches the CPML grows without bound within 300 steps at 64^3 on that
branch."""
import numpy as np
import pytest

from oracle import refcuda
from oracle.pyoracle import CpuSolver
from tests._util import rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcuda.available(), reason="oracle/_ref/libgsvit_refcuda.so not built")]

STEPS = 60


def test_reference_cuda_matches_the_oracle_in_vacuum(tmp_path):
    s = refcuda._scene("vacuum", 32, STEPS + 2, True, (91, 181))
    fout = str(tmp_path / "out.npz")
    d = refcuda.run("vacuum", 32, STEPS, 0, out_npz=fout, timeout=600)
    assert d["finite"] and d["steps"] == STEPS
    z = np.load(fout)
    got = [z[f"arr_{c}"] for c in range(6)]
    o = CpuSolver(s)
    o.step(STEPS)
    ref = o.fields()
    assert max(np.abs(x).max() for x in ref[:3]) > 0, "the TSF pulse has not entered the grid"
    errs = [rel_l2(a, b) for a, b in zip(got, ref)]
    print("reference CUDA vs oracle", ["%.2e" % e for e in errs], "%.3f ms/step" % d["ms_per_step"])
    assert max(errs) < 2e-4, errs
