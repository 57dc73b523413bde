"""Float form y = diag(s) W_q x (BF16 x, FP32 accumulation) and its backward
dx = W_q^T (s . dy), against a dense FP64 oracle and FP64 central finite
differences.  Errors are stated per output and bounded at 1e-2 relative for the
backward as specified; the observed errors are far smaller."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import ops
    from matvans_b200.autograd import Q8Linear, q8_linear


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


def bf16(rng, shape):
    return torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(torch.bfloat16)


def rel_err_per_output(got, ref, scale):
    """|got - ref| / sum of the magnitudes of the terms of each output."""
    return np.abs(got - ref) / np.maximum(scale, 1e-30)


@pytest.mark.parametrize("shape", [(256, 512), (4096, 11008), (11008, 4096)])
@pytest.mark.parametrize("B", [1, 8, 64])
def test_forward_and_backward_vs_fp64(shape, B):
    if shape != (256, 512) and B == 64 and shape[0] * shape[1] > 40_000_000:
        B = 64  # full config-4 sizes included
    rng = np.random.default_rng(hash((shape, B)) % 2 ** 32)
    W = gauss(rng, 4.0, shape)
    s = rng.uniform(1e-3, 1e-2, size=shape[0]).astype(np.float32)
    M = ops.Q8Matrix.encode(W, local=True)
    X = bf16(rng, (B, shape[1]))
    dY = bf16(rng, (B, shape[0]))
    st = torch.from_numpy(s)
    Y = M.matvec_bf16(X.cuda(), st).cpu().numpy().astype(np.float64)
    dX = M.matvec_t_bf16(dY.cuda(), st).cpu().numpy().astype(np.float64)
    W64, s64 = W.astype(np.float64), s.astype(np.float64)
    X64, dY64 = X.float().numpy().astype(np.float64), dY.float().numpy().astype(np.float64)
    Yref = (X64 @ W64.T) * s64[None, :]
    mag = (np.abs(X64) @ np.abs(W64).T) * s64[None, :]
    err_f = rel_err_per_output(Y, Yref, mag)
    dXref = (dY64 * s64[None, :]) @ W64
    magb = (np.abs(dY64) * s64[None, :]) @ np.abs(W64)
    err_b = rel_err_per_output(dX, dXref, magb)
    assert err_f.max() < 1e-5, err_f.max()
    assert err_b.max() < 1e-2 and np.median(err_b) < 1e-5, (err_b.max(), np.median(err_b))
    assert ops.device_status() == 0


def test_backward_matches_fp64_central_finite_differences():
    rng = np.random.default_rng(2026)
    W = gauss(rng, 4.0, (256, 512))
    s = rng.uniform(1e-3, 1e-2, size=256).astype(np.float32)
    M = ops.Q8Matrix.encode(W, local=True)
    B = 8
    X64 = rng.standard_normal((B, 512))
    R = bf16(rng, (B, 256))  # upstream gradient, exactly representable in bf16
    R64 = R.float().numpy().astype(np.float64)
    W64, s64 = W.astype(np.float64), s.astype(np.float64)

    def f(X):  # FP64 forward of the float form, contracted with R
        return float(np.sum(((X @ W64.T) * s64[None, :]) * R64))

    dX = M.matvec_t_bf16(R.cuda(), torch.from_numpy(s)).cpu().numpy().astype(np.float64)
    eps = 1e-3
    idx = [(int(b), int(c)) for b, c in zip(rng.integers(0, B, 64), rng.integers(0, 512, 64))]
    for b, c in idx:
        Xp, Xm = X64.copy(), X64.copy()
        Xp[b, c] += eps
        Xm[b, c] -= eps
        fd = (f(Xp) - f(Xm)) / (2 * eps)
        assert abs(dX[b, c] - fd) <= 1e-2 * max(abs(fd), 1e-3), (b, c, dX[b, c], fd)


def test_autograd_module():
    rng = np.random.default_rng(9)
    W = gauss(rng, 4.0, (384, 1024))
    s = rng.uniform(1e-3, 1e-2, size=384).astype(np.float32)
    layer = Q8Linear(W, s)
    x = bf16(rng, (4, 1024)).cuda().requires_grad_(True)
    y = layer(x)
    assert y.dtype == torch.float32 and y.shape == (4, 384)
    g = bf16(rng, (4, 384)).cuda().float()
    y.backward(g)
    ref = ((g.double().cpu().numpy() * s.astype(np.float64)[None, :]) @ W.astype(np.float64))
    got = x.grad.float().cpu().numpy()
    assert x.grad.dtype == torch.bfloat16
    assert np.allclose(got, ref, rtol=1e-2, atol=1e-2 * np.abs(ref).max())
    # functional form with an fp32 input is cast to bf16 on the way in
    y2 = q8_linear(x.detach().float(), layer.matrix, layer.scales)
    assert torch.allclose(y2, y.detach())
