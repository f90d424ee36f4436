"""The drop-in for GSvit's src3d/gpu.c refuses, at sv_gpu_new and before any
call into the library (so before any CUDA call), every deck that asks for
something the library does not step: outer boundaries other than CPML/none,
inner medium boundaries, non-TSF sources, subgrids, sums, forces, the
periodic far field and the RC dispersive material models.  GSvit's planned
structures are built on the CPU (oracle/_ref/libgsvit_dropin.so) and the GPU
branch is entered through sv_pool_allocate_gpus (pool.c:76-81); no GPU is
needed.  The library's thread-local last-error text is set to a marker first:
a refusal that reached the library would have replaced it."""
import ctypes as C

import pytest

from gsvit_copy_b200 import abi, plan
from tests import _dropin

pytestmark = pytest.mark.skipif(not _dropin.available(), reason="oracle/_ref/libgsvit_dropin.so not built")

FEATURES = [
    (0, "outer boundary other than CPML or none"),
    (1, "outer boundary other than CPML or none"),
    (2, "outer boundary other than CPML or none"),
    (3, "inner medium boundary"),
    (4, "point source"),
    (5, "SF source"),
    (6, "LTSF source"),
    (7, "TSFF source"),
    (8, "subgrid"),
    (9, "sum output"),
    (10, "force output"),
    (11, "periodic far field"),
    (12, "material type other than linear-tabulated"),
]


def _mark_last_error(lib):
    """Set the calling thread's last error to a known text (a NULL descriptor)."""
    h = C.c_void_p()
    assert lib.fdtd_plan_create(None, 0, C.byref(h)) != 0
    return lib.fdtd_last_error().decode()


@pytest.mark.parametrize("feature,words", FEATURES)
def test_dropin_refuses_before_any_library_call(feature, words, capfd):
    lib = abi.load_library()
    run = _dropin.DropinRun(plan.small_scene("ade", nsteps=8), gpu=True)
    marker = _mark_last_error(lib)
    assert marker
    assert run.lib.dropin_request(run.h, feature) == 0
    assert run.lib.dropin_start(run.h) == -1          # sv_gpu_new returned NULL
    err = capfd.readouterr().err
    assert "does not step this deck: unsupported " + words in err
    assert lib.fdtd_last_error().decode() == marker   # the library was never called


def test_supported_deck_reaches_the_library(capfd):
    """Control: without a request, sv_gpu_new goes on to fdtd_plan_create (which
    on a machine without a GPU fails with a CUDA error of its own)."""
    lib = abi.load_library()
    run = _dropin.DropinRun(plan.small_scene("ade", nsteps=8), gpu=True)
    marker = _mark_last_error(lib)
    rc = run.lib.dropin_start(run.h)
    assert "does not step this deck" not in capfd.readouterr().err
    assert rc == 0 or lib.fdtd_last_error().decode() != marker
