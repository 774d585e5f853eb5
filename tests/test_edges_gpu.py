"""Edge cases of the C ABI: oversized grids are refused before any
allocation or memory access (the output pointer is never touched), empty
batches and empty lookups are no-ops, and invalid Widom sizes are errors."""
import ctypes

import numpy as np
import pytest

import emptyroom_b200 as er
from emptyroom_b200 import _capi, synth

pytestmark = pytest.mark.gpu

ER_ERR_INVALID = 1
ER_ERR_LIMIT = 7


def _fw(ctx):
    f = synth.config1(2)
    return f, ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)


@pytest.mark.parametrize("flags", [er.ER_OUT_HOST, er.ER_OUT_HOST | er.ER_OUT_F64,
                                   er.ER_OUT_DEVICE | er.ER_OUT_F64])
def test_oversized_grid_refused_before_touching_output(ctx, flags):
    f, fw = _fw(ctx)
    small = np.zeros(8, dtype=np.float64)  # far smaller than the request
    st = _capi.lib().er_grid(ctx.handle, fw.id, 2000, 2000, 1001, flags,
                             small.ctypes.data_as(ctypes.c_void_p))
    assert st == ER_ERR_LIMIT
    assert not small.any()
    st = _capi.lib().er_grid(ctx.handle, fw.id, 1, 2000, 2000, flags,
                             small.ctypes.data_as(ctypes.c_void_p))
    assert st == ER_ERR_INVALID


def test_oversized_sheet_and_accessibility_refused(ctx):
    f, fw = _fw(ctx)
    sheet = np.zeros(8, dtype=np.float64)
    assert _capi.lib().er_grid_sheet(ctx.handle, fw.id, 2000, 2000, 1001, 0,
                                     sheet.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) \
        == ER_ERR_LIMIT
    acc = np.zeros(8, dtype=np.uint8)
    assert _capi.lib().er_accessibility(ctx.handle, fw.id, 2000, 2000, 1001,
                                        acc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))) \
        == ER_ERR_LIMIT
    assert not sheet.any() and not acc.any()


@pytest.mark.parametrize("mode", [er.ER_BATCH_PERSISTENT, er.ER_BATCH_PLAIN,
                                  er.ER_BATCH_PERSISTENT | er.ER_BATCH_HOST_OUT,
                                  er.ER_BATCH_PERSISTENT | er.ER_BATCH_COMP])
def test_empty_batch_is_a_no_op(ctx, mode):
    ctx.grid_batch([], mode)
    plan = ctx.batch_plan([], mode & ~er.ER_BATCH_HOST_OUT)
    plan.run()
    ctx.synchronize()
    plan.close()


def test_zero_point_lookup_and_widom_limits(ctx):
    import torch
    f, fw = _fw(ctx)
    g = torch.zeros((4, 4, 4), dtype=torch.float32, device="cuda")
    assert ctx.grid_interp(g.data_ptr(), (4, 4, 4), np.zeros((0, 3))).size == 0
    with pytest.raises(er.ErError):
        ctx.henry(fw, 298.0, 2**31, seed=0)
    with pytest.raises(er.ErError):
        ctx.henry(fw, float("nan"), 1000, seed=0)


def test_bounded_wait_gives_up_and_reports(ctx):
    """A kernel's bounded wait on a completion barrier that nothing completes
    gives up, raises the context's fault word, and the host sees it; the
    context then still computes (a small grid equals the one before)."""
    import numpy as np

    from emptyroom_b200 import _capi, synth
    f = synth.make_framework(6, (20.0, 20.0, 20.0), (90, 90, 90), 80)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    before = ctx.grid(fw, (9, 9, 9))
    st = _capi.lib().er_selftest_wait_timeout(ctx.handle, 4096)
    assert st == 0, _capi.lib().er_ctx_last_error(ctx.handle)
    assert np.array_equal(ctx.grid(fw, (9, 9, 9)), before)
    fw.release()
