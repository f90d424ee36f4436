"""fdtd_step_static_scratch, the step for callers that cannot call cudaMalloc
where they step (their device memory belongs to another allocator, or
cudaMalloc's device-wide synchronisation would stall other streams): its TSF
face tables live in a static device array.  Checked against fdtd_step through
the C ABI on two calls in a row.  Collected last on purpose, and it must give
the same bits whether it runs alone or after other plans in the process."""
import ctypes as C

import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from gsvit_copy_b200.solver import Solver
from tests._util import random_fields

pytestmark = pytest.mark.gpu


def _static_step(solver, n):
    abi.check(solver.lib.fdtd_step_static_scratch(solver.h, n), "fdtd_step_static_scratch")


@pytest.mark.parametrize("kind", ["full", "ade"])
def test_static_scratch_step_matches_step_on_two_calls(kind):
    s = plan.small_scene(kind, nsteps=80)
    ref, st = Solver(s), Solver(s)
    init = random_fields((s.xres, s.yres, s.zres), 21)
    ref.set_fields(init)
    st.set_fields(init)
    for _ in range(2):
        ref.step(35)
        _static_step(st, 35)
        for a, b in zip(ref.fields(), st.fields()):
            assert np.array_equal(a, b)
        assert np.array_equal(ref.probes(), st.probes())
        assert ref.step_count == st.step_count
    assert np.array_equal(ref.nfff_spectrum(), st.nfff_spectrum())
    ref.close()
    st.close()


def test_static_scratch_rejects_tables_above_the_limit():
    """A 1100 x 1100 x 8 grid whose TSF box has 2 x 1096^2 z-face cells needs
    more than the 32 MiB of static scratch: refused, state untouched."""
    dx = 10e-9
    dt = plan.plan_dt(dx, dx, dx, 0.5)
    s = plan.Scene(name="wide", xres=1100, yres=1100, zres=8, dx=dx, dt=dt, nsteps=4)
    s.mats = [plan.vacuum_material()]
    s.mat = np.zeros((1100, 1100, 8), dtype=np.int32)
    s.tsf = dict(box=((2, 2, 2), (1097, 1097, 5)), theta=0.3, phi=0.2, psi=0.1,
                 wave=plan.gaussian_pulse(5, dt, 20 * dx, 3 * dt, 2 * dt))
    nface = 2 * (1096 * 4 + 1096 * 4 + 1096 * 1096)
    assert nface * 2 * 8 > abi.STATIC_SCRATCH_BYTES
    g = Solver(s)
    g.step(1)
    before = g.fields(abi.E_ALL, dtype=np.float32)
    rc = g.lib.fdtd_step_static_scratch(g.h, 2)
    assert rc == -2
    assert "32 MiB" in g.lib.fdtd_last_error().decode()
    assert g.step_count == 1
    after = g.fields(abi.E_ALL, dtype=np.float32)
    for a, b in zip(before[:3], after[:3]):
        assert np.array_equal(a, b)
    g.close()
