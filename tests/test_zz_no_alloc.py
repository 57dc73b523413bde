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


_FRESH = r"""
import ctypes, sys
import numpy as np
import torch
from matvans_b200 import _lib

L = _lib.lib()
dev = torch.device("cuda", 0)
n = 50000
y = torch.from_numpy(np.random.default_rng(5).integers(-2**20, 2**20, size=n).astype(np.int32)).to(dev)
out = torch.empty(n, dtype=torch.int8, device=dev)
delta = torch.empty(1, dtype=torch.float32, device=dev)
stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

def call():
    _lib.check(L.mv_requant_absmax_noalloc(ctypes.c_void_p(y.data_ptr()), n, ctypes.c_void_p(out.data_ptr()),
                                           ctypes.c_void_p(delta.data_ptr()), stream))

def status_word():
    v = ctypes.c_uint64(7)
    _lib.check(L.mv_debug_query(1, ctypes.byref(v)))
    return v.value

torch.cuda.synchronize()
assert status_word() == 0, "status word exists before any call"
call()  # the first call loads the library's kernels and looks up the scratch array's address
torch.cuda.synchronize()
free0, _ = torch.cuda.mem_get_info()
reserved0 = torch.cuda.memory_reserved()
for _ in range(5):
    call()
torch.cuda.synchronize()
free1, _ = torch.cuda.mem_get_info()
assert status_word() == 0, "the allocation-free path created the status word"
assert torch.cuda.memory_reserved() == reserved0, "torch's allocator grew"
assert free1 == free0, f"device memory in use grew by {free0 - free1} bytes"
d = np.float32(np.float32(np.abs(y.cpu().numpy().astype(np.int64)).max()) / np.float32(127))
assert np.float32(delta.item()) == d
print("ok")
"""


def test_noalloc_allocates_nothing_in_a_fresh_process():
    """In a process that has called nothing else in the library, the allocation-free entry point creates no
    device memory: the library's lazily created status word stays absent, torch's caching allocator does not
    grow, and the device's free memory is unchanged across repeated calls."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]
