"""The bounded-wait error path of the TMA tile kernels, made to run out on the
GPU without a fault: GSVIT_B200_STALL_TEST makes every tile CTA of a plan
created while it is set also wait, for a few polls, on an mbarrier that
nothing arrives on.  The CTA then sets the plan's error word, drains its TMA
copies (full-length bounded waits on the real barriers) and returns, so the
context stays usable.  The host must report FDTD_E_TIMEOUT on sync and on
every readback, refuse further steps, and a fresh plan must then step
bit-exact."""
import numpy as np
import pytest

from gsvit_copy_b200 import abi, plan
from gsvit_copy_b200.solver import Solver
from tests._util import random_fields

pytestmark = pytest.mark.gpu


def _code(fn):
    try:
        fn()
    except abi.FdtdError as e:
        return str(e)
    return ""


def test_expired_wait_is_reported_and_plan_is_refused(monkeypatch):
    monkeypatch.setenv("GSVIT_B200_TILES", "1")   # the stall hook lives in the tile kernels
    s = plan.small_scene("full", nsteps=16)
    init = random_fields((s.xres, s.yres, s.zres), 9)
    ref = Solver(s)                    # created without the stall
    ref.set_fields(init)
    ref.step(4)
    want = ref.fields(dtype=np.float32)

    monkeypatch.setenv("GSVIT_B200_STALL_TEST", "64")
    bad = Solver(s)
    monkeypatch.delenv("GSVIT_B200_STALL_TEST")
    bad.set_fields(init)
    bad.step(1)                        # launches return; the CTAs give up on the device
    assert "timeout" in _code(bad.sync).lower()
    assert "timeout" in _code(lambda: bad.fields(dtype=np.float32)).lower()
    assert "state" in _code(lambda: bad.step(1)).lower()
    bad.close()

    fresh = Solver(s)
    fresh.set_fields(init)
    fresh.step(4)
    for a, b in zip(fresh.fields(dtype=np.float32), want):
        assert np.array_equal(a, b)
