"""The C ABI rejects bad arguments itself, before it touches the GPU: every
call below returns MV_ERR_ARG or MV_ERR_SHAPE with a message, on a machine
without a CUDA device (a CUDA call would have returned MV_ERR_CUDA).  The
device pointers are stand-ins that the library never dereferences on these
paths."""
import ctypes

import pytest

from matvans_b200 import _lib
from matvans_b200._lib import Q8StackInfo, Q8Tuning, Q8View

MV_ERR_ARG, MV_ERR_SHAPE, MV_ERR_CUDA = 1, 2, 5
FAKE = 0x10000  # 16-byte aligned stand-in for a device pointer


def _view(rows=64, cols=512, seg_quads=16, local=1):
    v = Q8View()
    v.blocks = v.blk_off = v.tbl = v.tbl_off = FAKE
    v.rows, v.cols, v.seg_quads, v.local = rows, cols, seg_quads, local
    v.nseg = -(-(cols // 4) // seg_quads)
    v.max_blk_rows, v.blocks_rows, v.tbl_len, v.tbl_stripe_max = 4, 1024, 1024, 64
    return v


def _expect(rc, code, words):
    L = _lib.lib()
    msg = L.mv_last_error().decode()
    assert rc == code, (rc, msg)
    assert words in msg, msg


def test_noalloc_requant_rejects_null_and_oversized_inputs():
    L = _lib.lib()
    _expect(L.mv_requant_absmax_noalloc(None, 16, None, None, None), MV_ERR_ARG, "bad arguments")
    _expect(L.mv_requant_absmax_noalloc(FAKE, 0, FAKE, None, None), MV_ERR_ARG, "bad arguments")
    # one element beyond the static scratch's limit
    _expect(L.mv_requant_absmax_noalloc(FAKE, 33554433, FAKE, None, None), MV_ERR_ARG, "static scratch limit")


def test_stack_launch_rejects_bad_batch_and_missing_jobs():
    L = _lib.lib()
    info, t = Q8StackInfo(), Q8Tuning(8, 1, 1, 0, 0, 0)
    _expect(L.mv_q8_stack_matvec(None, 1, ctypes.byref(info), 1, ctypes.byref(t), None), MV_ERR_ARG, "batch must be")
    for batch in (0, 17):
        _expect(L.mv_q8_stack_matvec(FAKE, 1, ctypes.byref(info), batch, ctypes.byref(t), None), MV_ERR_ARG,
                "batch must be 1..16")
    # the launch's tuning must be the one the jobs were planned with
    info.warps, info.ilp = 4, 1
    _expect(L.mv_q8_stack_matvec(FAKE, 1, ctypes.byref(info), 4, ctypes.byref(t), None), MV_ERR_ARG,
            "tuning differs")


@pytest.mark.parametrize("cols,x,seg_quads", [(100, FAKE, 16), (512, FAKE + 4, 16), (512, FAKE, 6)])
def test_tuned_q8_launch_rejects_layouts_it_cannot_take(cols, x, seg_quads):
    L = _lib.lib()
    v = _view(cols=cols, seg_quads=seg_quads)
    _expect(L.mv_q8_matvec_tuned(ctypes.byref(v), x, 1, FAKE, None, None, None, None), MV_ERR_ARG, "needs cols")
    _expect(L.mv_q8_matvec_bf16(ctypes.byref(v), x, 1, FAKE, FAKE, None, None), MV_ERR_ARG, "needs cols")


def test_q8_launches_reject_null_buffers():
    L = _lib.lib()
    v = _view()
    _expect(L.mv_q8_matvec_tuned(None, FAKE, 1, FAKE, None, None, None, None), MV_ERR_ARG, "bad arguments")
    _expect(L.mv_q8_matvec_tuned(ctypes.byref(v), FAKE, 0, FAKE, None, None, None, None), MV_ERR_ARG,
            "bad arguments")
    _expect(L.mv_q8_matvec_tuned(ctypes.byref(v), FAKE, 1, FAKE, None, FAKE, None, None), MV_ERR_ARG,
            "needs scales")
    _expect(L.mv_q8_matvec_bf16(ctypes.byref(v), None, 1, FAKE, FAKE, None, None), MV_ERR_ARG, "bad arguments")
    rc = L.mv_q8_matvec(ctypes.byref(v), None, 1, FAKE, None, None, None)
    assert rc == MV_ERR_ARG, L.mv_last_error()


def test_dense_comparator_checks_shape_and_alignment():
    L = _lib.lib()
    _expect(L.mv_dense_matvec(None, 4, 16, FAKE, 1, FAKE, None), MV_ERR_ARG, "bad arguments")
    _expect(L.mv_dense_matvec(FAKE, 4, 100, FAKE, 1, FAKE, None), MV_ERR_SHAPE, "cols % 16")
    _expect(L.mv_dense_matvec(FAKE + 8, 4, 16, FAKE, 1, FAKE, None), MV_ERR_ARG, "16-byte aligned")


def test_reference_layout_kernels_reject_null_streams():
    L = _lib.lib()
    rc = L.mv_awr_matvec(None, 0, None, None, None, None, 32, 128, None, 1, None, None, None, None)
    assert rc == MV_ERR_ARG, L.mv_last_error()
    rc = L.mv_aws_matvec(None, 0, None, None, None, None, 32, 128, None, 1, None, None, None, None)
    assert rc == MV_ERR_ARG, L.mv_last_error()
    for rc in (L.mv_awr_matvec(FAKE, 64, FAKE, FAKE, FAKE, FAKE, 32, 100, FAKE, 1, FAKE, None, None, None),
               L.mv_aws_matvec(FAKE, 64, FAKE, FAKE, FAKE, FAKE, 33, 128, FAKE, 1, FAKE, None, None, None)):
        assert rc == MV_ERR_SHAPE, L.mv_last_error()
