"""Float form on the tensor cores (kind::f16 MMAs, engine 0) against the dense
FP64 oracle and against the CUDA-core engine (engine 1): batches that fill,
split and straddle the 16-vector forward and 32-vector backward passes,
segment lengths that leave half-filled 8-quad pieces, ragged shapes, global and
per-row tables.  The error of each output is stated relative to the sum of the
magnitudes of its terms (the same measure as the other float-form tests)."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import ops

MMA, CUDA_CORES = 0, 1
FWD_TOL = 1e-5   # max over outputs, forward (exact products, fp32 accumulation)
BWD_TOL = 1e-4   # max over outputs, backward (s . dy carried as a bf16 hi/lo pair, ~2^-17 relative)


@pytest.fixture(autouse=True)
def clean_status():
    ops.device_status(raise_on_error=False)
    yield


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


def bf16(rng, shape):
    return torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(torch.bfloat16)


def run_case(W, s, B, rng, seg_quads=0, local=True, warps=4):
    M = ops.Q8Matrix.encode(W, local=local, seg_quads=seg_quads)
    X, dY = bf16(rng, (B, W.shape[1])), bf16(rng, (B, W.shape[0]))
    st = torch.from_numpy(s)
    W64, s64 = W.astype(np.float64), s.astype(np.float64)
    X64, dY64 = X.float().numpy().astype(np.float64), dY.float().numpy().astype(np.float64)
    Yref = (X64 @ W64.T) * s64[None, :]
    magf = (np.abs(X64) @ np.abs(W64).T) * s64[None, :]
    dXref = (dY64 * s64[None, :]) @ W64
    magb = (np.abs(dY64) * s64[None, :]) @ np.abs(W64)
    out = {}
    for eng in (MMA, CUDA_CORES):
        t = (warps, 1, 1, 0, 0, eng)
        Y = M.matvec_bf16(X.cuda(), st, tuning=t).cpu().numpy().astype(np.float64)
        dX = M.matvec_t_bf16(dY.cuda(), st, tuning=t).cpu().numpy().astype(np.float64)
        ef = (np.abs(Y - Yref) / np.maximum(magf, 1e-30)).max()
        eb = (np.abs(dX - dXref) / np.maximum(magb, 1e-30)).max()
        assert ef < FWD_TOL, (eng, B, ef)
        assert eb < BWD_TOL, (eng, B, eb)
        out[eng] = (Y, dX)
    assert ops.device_status() == 0
    return out


@pytest.mark.parametrize("B", [2, 7, 16, 17, 32, 33, 64])
def test_float_mma_batches(B):
    rng = np.random.default_rng(100 + B)
    W = gauss(rng, 4.0, (256, 512))
    s = rng.uniform(1e-3, 1e-2, size=256).astype(np.float32)
    run_case(W, s, B, rng)


@pytest.mark.parametrize("seg_quads", [8, 36, 44, 64, 128])
@pytest.mark.parametrize("local", [True, False])
def test_float_mma_segments_and_ragged_rows(seg_quads, local):
    rng = np.random.default_rng(seg_quads + 7 * local)
    W = gauss(rng, 3.0, (100, 1520))
    s = rng.uniform(1e-3, 1e-2, size=100).astype(np.float32)
    for warps in (1, 3, 8):
        run_case(W, s, 9, rng, seg_quads=seg_quads, local=local, warps=warps)


def test_float_mma_extreme_values():
    rng = np.random.default_rng(9)
    W = np.where(rng.random((64, 2048)) < 0.5, -127, 127).astype(np.int8)
    s = np.full(64, 1e-2, np.float32)
    run_case(W, s, 16, rng, local=False)
    Z = np.zeros((64, 512), np.int8)
    run_case(Z, s, 5, rng)
