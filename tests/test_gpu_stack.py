"""Persistent Q8 kernel: every launch-parameter combination and the batched
(many matrices, one launch) form, bit-exact against the CPU oracle."""
import numpy as np
import pytest

from conftest import cuda_ok
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import ops, _lib


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


@pytest.fixture(autouse=True)
def clean_status():
    ops.device_status(raise_on_error=False)
    yield


TUNINGS = [(w, ilp, d, 0) for w in (1, 4, 8) for ilp in (1, 2) for d in (1, 2)] + \
    [(8, 2, 1, 1), (3, 2, 2, 2), (8, 1, 2, 0, 3), (4, 2, 2, 0, 1), (2, 1, 1, 0, 5)]


@pytest.mark.parametrize("tuning", TUNINGS)
def test_q8_persistent_all_tunings(tuning):
    rng = np.random.default_rng(sum(tuning))
    for shape, local in (((100, 1008), True), ((257, 2048), False), ((64, 4096), True)):
        W = gauss(rng, 3.0, shape)
        M = ops.Q8Matrix.encode(W, local=local)
        for B in (1, 3, 8, 16, 20):
            x = rng.integers(-127, 128, size=(B, shape[1])).astype(np.int8)
            s = rng.uniform(1e-3, 1e-2, size=shape[0]).astype(np.float32)
            y, ys = M.matvec(torch.from_numpy(x), scales=s, tuning=tuning)
            yref = oracle.matvec_i8(W, x)
            assert np.array_equal(y.cpu().numpy(), yref), (shape, B)
            assert np.array_equal(ys.cpu().numpy(), (yref.astype(np.float32) * s[None, :]).astype(np.float32))
    assert ops.device_status() == 0


def test_q8_tuned_rejects_unsupported_shapes():
    W = np.zeros((64, 1000), np.int8)
    M = ops.Q8Matrix.encode(W)
    with pytest.raises(_lib.MatvansError):
        M.matvec(torch.zeros((1, 1000), dtype=torch.int8), tuning=(8, 2, 1, 0))
    # the default entry point falls back to the general kernel for the same matrix
    assert M.matvec(torch.ones((1, 1000), dtype=torch.int8)).abs().sum().item() == 0


def test_q8_stack_uneven_shapes_one_launch():
    rng = np.random.default_rng(42)
    shapes = [(512, 512), (1376, 512), (512, 1376), (96, 4096), (4096, 96), (33, 208)]
    Ws, Ms = [], []
    for i, sh in enumerate(shapes):
        if i % 3 == 2:  # Laplace with rare +-100 outliers
            W = np.clip(np.round(rng.laplace(0, 3, sh)), -127, 127).astype(np.int8)
            mask = rng.random(sh) < 0.001
            W[mask] = rng.choice(np.array([-100, 100], np.int8), size=mask.sum())
        else:
            W = gauss(rng, rng.uniform(2, 6), sh)
        Ws.append(W)
        Ms.append(ops.Q8Matrix.encode(W, local=(i % 2 == 0)))
    for B in (1, 4, 8, 16):
        for tuning in ((0, 0, 0, 0), (4, 1, 2, 0), (8, 2, 2, 0, 2)):
            xs = [torch.from_numpy(rng.integers(-127, 128, size=(B, M.cols)).astype(np.int8)).cuda() for M in Ms]
            sc = [torch.from_numpy(rng.uniform(1e-3, 1e-2, size=M.rows).astype(np.float32)).cuda() for M in Ms]
            S = ops.Q8Stack(Ms, batch=B, tuning=tuning, xs=xs, scales=sc)
            ys = S.run()
            for W, x, y, yscaled, s in zip(Ws, xs, ys, S.yss, sc):
                yref = oracle.matvec_i8(W, x.cpu().numpy())
                assert np.array_equal(y.cpu().numpy(), yref), (W.shape, B, tuning)
                sref = (yref.astype(np.float32) * s.cpu().numpy()[None, :]).astype(np.float32)
                assert np.array_equal(yscaled.cpu().numpy(), sref)
    assert ops.device_status() == 0


def test_q8_stack_graph_replay():
    rng = np.random.default_rng(7)
    Ws = [gauss(rng, 4, (256, 1024)), gauss(rng, 2, (1024, 256))]
    Ms = [ops.Q8Matrix.encode(W, local=True) for W in Ws]
    S = ops.Q8Stack(Ms, batch=2)
    S.run()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        S.run()
    torch.cuda.current_stream().wait_stream(s)
    with torch.cuda.graph(g):
        S.run()
    for trial in range(3):
        xs = [rng.integers(-127, 128, size=(2, M.cols)).astype(np.int8) for M in Ms]
        for xd, xh in zip(S.xs, xs):
            xd.copy_(torch.from_numpy(xh))
        g.replay()
        torch.cuda.synchronize()
        for W, xh, y in zip(Ws, xs, S.ys):
            assert np.array_equal(y.cpu().numpy(), oracle.matvec_i8(W, xh))
    del g
    assert ops.device_status() == 0
