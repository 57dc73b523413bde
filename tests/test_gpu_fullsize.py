"""Full-size parity of the batched and large-matrix configurations, against the oracle.

* The batched uneven stack: two transformer layers of q,k,v,o (4096x4096), gate, up (11008x4096) and down
  (4096x11008), per-row tables, each matrix with its own sigma in [2, 6] and two of them Laplace(b=3) with
  0.1 % of entries at +-100, in ONE persistent launch, at 1, 4, 8 and 16 vectors (16 runs on the tensor
  cores), every output row checked.
* The large low-entropy matrix: 16384x16384 with Laplace(b=2) weights and per-row tables, 1 and 16 vectors,
  checked on a sample of 2048 rows (every 8th) against the oracle's int64 product of those rows.

The oracle's int8 matvec does not depend on the codec, so these are checks of the decode, not of one kernel
against another.
"""
import numpy as np
import pytest

from conftest import cuda_ok
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import ops

LAYER = [("q", 4096, 4096), ("k", 4096, 4096), ("v", 4096, 4096), ("o", 4096, 4096),
         ("gate", 11008, 4096), ("up", 11008, 4096), ("down", 4096, 11008)]


def stack_weights(rng, layers=2):
    n = layers * len(LAYER)
    laplace = {3, 11}  # one matrix per layer
    out = []
    for i in range(n):
        _, r, c = LAYER[i % len(LAYER)]
        if i in laplace:
            z = rng.laplace(0.0, 3.0, size=(r, c)).astype(np.float32)
            u = rng.random((r, c), dtype=np.float32)
            z[u < 0.0005] = -100.0
            z[(u >= 0.0005) & (u < 0.001)] = 100.0
        else:
            z = rng.standard_normal((r, c), dtype=np.float32) * np.float32(rng.uniform(2, 6))
        out.append(np.clip(np.rint(z), -127, 127).astype(np.int8))
    return out


def test_full_stack_two_layers_all_batches():
    rng = np.random.default_rng(2024)
    Ws = stack_weights(rng)
    Ms = [ops.Q8Matrix.encode(W, local=True) for W in Ws]
    for B in (1, 4, 8, 16):
        xs = [torch.from_numpy(rng.integers(-127, 128, size=(B, W.shape[1])).astype(np.int8)).cuda() for W in Ws]
        S = ops.Q8Stack(Ms, batch=B, xs=xs)
        S.run()
        torch.cuda.synchronize()
        ops.device_status()
        for i, (W, x, y) in enumerate(zip(Ws, xs, S.ys)):
            ref = oracle.matvec_i8(W, x.cpu().numpy())
            assert np.array_equal(y.cpu().numpy(), ref), f"matrix {i} at B={B}"


def test_large_16384_laplace_sampled_rows():
    rng = np.random.default_rng(2025)
    n = 16384
    W = np.empty((n, n), np.int8)
    for r0 in range(0, n, 1024):  # in row blocks: the float draws of the whole matrix would take 2 GB
        W[r0:r0 + 1024] = np.clip(np.rint(rng.laplace(0.0, 2.0, size=(1024, n))), -127, 127).astype(np.int8)
    M = ops.Q8Matrix.encode(W, local=True)
    rows = np.arange(0, n, 8)
    Ws = np.ascontiguousarray(W[rows])
    for B in (1, 16):
        x = rng.integers(-127, 128, size=(B, n)).astype(np.int8)
        y = M.matvec(torch.from_numpy(x).cuda())
        torch.cuda.synchronize()
        ops.device_status()
        assert np.array_equal(y.cpu().numpy()[:, rows], oracle.matvec_i8(Ws, x)), f"B={B}"
