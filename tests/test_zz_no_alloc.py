"""The allocation-free requantisation entry point against the scratch-taking one.

mv_requant_absmax_noalloc exists for callers that cannot allocate device memory
(for example a plugin whose host framework owns the allocator, or a latency path
that cannot take cudaMalloc's implicit synchronisation).  It must give exactly the results of
mv_requant_absmax, which takes caller-owned scratch, on consecutive calls that
reuse its static scratch array.  Called through the C ABI.
"""
import ctypes

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]


def test_noalloc_requant_matches_scratch_version_on_two_calls():
    import torch
    from matvans_b200 import _lib

    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(31)
    # two consecutive calls with different data: the second must not see the first's scratch
    for n, scale in ((20000, 2 ** 20), (70001, 2 ** 24)):
        y = torch.from_numpy(rng.integers(-scale, scale, size=n).astype(np.int32)).cuda()
        out_ref = torch.empty(n, dtype=torch.int8, device="cuda")
        out_new = torch.empty(n, dtype=torch.int8, device="cuda")
        d_ref = torch.empty(1, dtype=torch.float32, device="cuda")
        d_new = torch.empty(1, dtype=torch.float32, device="cuda")
        scratch = torch.empty(1, dtype=torch.int32, device="cuda")
        _lib.check(L.mv_requant_absmax(ctypes.c_void_p(y.data_ptr()), n, ctypes.c_void_p(out_ref.data_ptr()),
                                       ctypes.c_void_p(d_ref.data_ptr()), ctypes.c_void_p(scratch.data_ptr()),
                                       stream))
        _lib.check(L.mv_requant_absmax_noalloc(ctypes.c_void_p(y.data_ptr()), n,
                                               ctypes.c_void_p(out_new.data_ptr()),
                                               ctypes.c_void_p(d_new.data_ptr()), stream))
        torch.cuda.synchronize()
        assert torch.equal(out_new, out_ref)
        assert d_new.item() == d_ref.item()
        # the result itself: delta = max|y| / 127 in fp32, out = rn(y / delta)
        yh = y.cpu().numpy()
        d = np.float32(np.float32(np.abs(yh.astype(np.int64)).max()) / np.float32(127))
        assert np.float32(d_new.item()) == d
        assert np.array_equal(out_new.cpu().numpy(), np.rint(yh.astype(np.float32) / d).astype(np.int8))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from matvans_b200 import _lib

    L = _lib.lib()
    y = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.empty(16, dtype=torch.int8, device="cuda")
    rc = L.mv_requant_absmax_noalloc(ctypes.c_void_p(y.data_ptr()), 33554433, ctypes.c_void_p(out.data_ptr()),
                                     None, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 1 and b"static scratch limit" in L.mv_last_error()
