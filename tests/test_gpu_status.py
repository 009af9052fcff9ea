"""Bounded device waits and the plan's status word.

The slab and plane passes wait on mbarriers for their bulk copies with an
iteration limit; a wait that runs out stores an error code into the plan's
status word (mapped host memory) instead of spinning.  The next compute call
on the plan reports it once as SFL_ERR_TIMEOUT.  The failure is made without
any copy in flight: sfl_plan_selftest_wait runs one wait, with a short limit,
on an mbarrier that nothing completes.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def status(sfl, ws, reset=0):
    st = C.c_int32(-1)
    assert sfl.lib.sfl_plan_status(ws._h, C.byref(st), reset) == 0
    return st.value


@pytest.mark.parametrize("pipeline", ["slabs", "lines"])
def test_timed_out_wait_is_reported_once_by_the_next_call(sfl, pipeline):
    dims = (64, 64, 64)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 2], bernstein_order=6)
    ws = sfl.make_workspace(t, "float32", dims)
    ws.set_pipeline(pipeline)
    x = sfl.to_device(np.random.default_rng(3).standard_normal(dims).astype(np.float32))
    c0 = sfl.analyze(ws, x)
    assert status(sfl, ws) == 0
    assert sfl.lib.sfl_plan_selftest_wait(ws._h, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    assert status(sfl, ws) == 1                 # recorded (synchronizes), not cleared
    with pytest.raises(sfl.DeviceWaitTimeout, match="bounded device wait"):
        sfl.analyze(ws, x)
    assert status(sfl, ws) == 0                 # reported once
    c1 = sfl.analyze(ws, x)                     # the plan works on
    assert torch.equal(c0, c1)
    # cleared by the status query instead
    sfl.lib.sfl_plan_selftest_wait(ws._h, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert status(sfl, ws, reset=1) == 1
    assert torch.equal(sfl.synthesize(ws, c1), sfl.synthesize(ws, c0))


def test_selftest_needs_an_ns_plan(sfl):
    ws = sfl.make_workspace(sfl.Surfacelet(scales=1, direction_levels=[1]), "float32", (48, 48, 48))
    rc = sfl.lib.sfl_plan_selftest_wait(ws._h, None)
    assert rc == sfl._lib.SFL_ERR_ARGUMENT
