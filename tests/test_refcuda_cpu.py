"""GSvit's own CUDA path as built here (oracle/_ref/libgsvit_refcuda.so, the
measured context baseline): on a machine without a GPU the library loads,
exports the driver's entry points, and a run fails loudly -- the
reference's sv_gpu_new finds no device and the driver refuses the plan
instead of timing an empty loop."""
import ctypes as C

import pytest

from oracle import refcuda

pytestmark = pytest.mark.skipif(not refcuda.available(), reason="oracle/_ref/libgsvit_refcuda.so not built")


def test_library_exports_the_driver_and_gsvit_gpu_entry_points():
    lib = C.CDLL(refcuda.REFCUDA_SO)
    for name in ("ref_create", "dropin_start", "dropin_step", "dropin_finish", "sv_gpu_new",
                 "sv_pool_gpu_ystep_h", "sv_pool_gpu_copyfrom", "wrap_eKernel", "g_queue_new", "g_thread_create"):
        assert hasattr(lib, name), name


def test_run_without_a_device_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="sv_gpu_new"):
        refcuda.run("vacuum", 16, steps=2, warmup=0, timeout=300)
