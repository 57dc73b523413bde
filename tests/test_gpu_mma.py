"""Tensor-core (tcgen05.mma kind::i8) consumer of the persistent Q8 kernel:
3..16 int8 vectors (multiplied 16 wide, the missing ones zero), exact int32
accumulation in tensor memory.  Every case is
compared bit for bit with the CPU oracle and with the CUDA-core dp4a engine
on the same launch parameters."""
import numpy as np
import pytest

from conftest import cuda_ok
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import ops, _lib

MMA, DP4A = 0, 1


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


@pytest.fixture(autouse=True)
def clean_status():
    ops.device_status(raise_on_error=False)
    yield


def _both_engines(M, W, x, s, tuning):
    t = tuple(tuning) + (0,) * (5 - len(tuning))
    xt = torch.from_numpy(x)
    y0, ys0 = M.matvec(xt, scales=s, tuning=t + (MMA,))
    # the CUDA-core engine takes at most 8 warps per CTA
    y1, ys1 = M.matvec(xt, scales=s, tuning=(min(t[0], 8),) + t[1:] + (DP4A,))
    yref = oracle.matvec_i8(W, x)
    assert np.array_equal(y0.cpu().numpy(), yref)
    assert np.array_equal(y1.cpu().numpy(), yref)
    sref = (yref.astype(np.float32) * s[None, :]).astype(np.float32)
    assert np.array_equal(ys0.cpu().numpy(), sref)


@pytest.mark.parametrize("B", [3, 4, 5, 8, 9, 12, 15, 16])
@pytest.mark.parametrize("local", [True, False])
def test_mma_batches(B, local):
    rng = np.random.default_rng(B + 100 * local)
    for shape in ((64, 512), (100, 1008), (257, 2048)):
        W = gauss(rng, 4.0, shape)
        M = ops.Q8Matrix.encode(W, local=local)
        x = rng.integers(-127, 128, size=(B, shape[1])).astype(np.int8)
        s = rng.uniform(1e-3, 1e-2, size=shape[0]).astype(np.float32)
        _both_engines(M, W, x, s, (4, 1, 1, 0))
    assert ops.device_status() == 0


# segment lengths that leave a half-filled 8-quad chunk (36, 44) or a short last segment
@pytest.mark.parametrize("seg_quads", [8, 36, 44, 64, 128])
def test_mma_segment_lengths(seg_quads):
    rng = np.random.default_rng(seg_quads)
    W = gauss(rng, 3.0, (96, 1520))
    M = ops.Q8Matrix.encode(W, local=True, seg_quads=seg_quads)
    x = rng.integers(-127, 128, size=(16, 1520)).astype(np.int8)
    s = rng.uniform(1e-3, 1e-2, size=96).astype(np.float32)
    tunings = [(1, 1, 1, 0), (4, 1, 2, 0), (8, 1, 1, 0, 3), (3, 1, 2, 2)]
    if seg_quads <= 64:  # 8 warps of two 128-quad stream buffers exceed shared memory (rejected, tested below)
        # 16 warps: warps 8..15 keep their x tiles outside the decode table's holes
        tunings += [(8, 1, 2, 0), (6, 1, 2, 0, 2), (16, 1, 1, 0), (12, 1, 1, 0, 2)]
    for tuning in tunings:
        _both_engines(M, W, x, s, tuning)
    assert ops.device_status() == 0


def test_launches_that_do_not_fit_are_rejected():
    M = ops.Q8Matrix.encode(np.ones((64, 512), np.int8))
    with pytest.raises(_lib.MatvansError):  # the CUDA-core float backward takes at most 8 warps per CTA
        M.matvec_t_bf16(torch.ones((1, 64), dtype=torch.bfloat16, device="cuda"),
                        torch.ones(64, device="cuda"), tuning=(16, 1, 1, 0, 0, DP4A))
    W = np.random.default_rng(1).integers(-127, 128, size=(96, 1520)).astype(np.int8)  # ~8 bits/weight
    M = ops.Q8Matrix.encode(W, local=True, seg_quads=128)
    with pytest.raises(_lib.MatvansError):  # 8 warps of two 128-quad stream buffers exceed shared memory
        M.matvec(torch.ones((16, 1520), dtype=torch.int8), tuning=(8, 1, 2, 0, 0, MMA))
    with pytest.raises(_lib.MatvansError):  # so do 16 warps of one 128-quad stream buffer each
        M.matvec(torch.ones((16, 1520), dtype=torch.int8), tuning=(16, 1, 1, 0, 0, MMA))
    assert ops.device_status() == 0


def test_mma_extreme_values():
    # |y| up to 127 * 127 * cols: exact in int32 for these widths
    rng = np.random.default_rng(5)
    W = np.where(rng.random((64, 4096)) < 0.5, -127, 127).astype(np.int8)
    M = ops.Q8Matrix.encode(W, local=False)
    x = np.full((16, 4096), -127, np.int8)
    x[1::2] = 127
    s = np.ones(64, np.float32)
    _both_engines(M, W, x, s, (4, 1, 1, 0))
    Z = np.zeros((64, 1024), np.int8)
    M = ops.Q8Matrix.encode(Z, local=True)
    x = rng.integers(-127, 128, size=(8, 1024)).astype(np.int8)
    _both_engines(M, Z, x, s, (8, 1, 1, 0))
    assert ops.device_status() == 0


def test_mma_large_batch_passes():
    # batches above 16 run in passes of 16; the last pass (here 4 or 9 vectors) picks its engine itself
    rng = np.random.default_rng(11)
    W = gauss(rng, 4.0, (200, 1024))
    M = ops.Q8Matrix.encode(W, local=True)
    for B in (20, 25, 48):
        x = rng.integers(-127, 128, size=(B, 1024)).astype(np.int8)
        y = M.matvec(torch.from_numpy(x))
        assert np.array_equal(y.cpu().numpy(), oracle.matvec_i8(W, x))
    assert ops.device_status() == 0


@pytest.mark.parametrize("engine", [MMA, DP4A])
def test_mma_stack(engine):
    rng = np.random.default_rng(3 + engine)
    shapes = [(512, 512), (1376, 512), (512, 1376), (96, 4096), (33, 208)]
    Ws = [gauss(rng, rng.uniform(2, 6), sh) for sh in shapes]
    Ms = [ops.Q8Matrix.encode(W, local=(i % 2 == 0)) for i, W in enumerate(Ws)]
    for B in (3, 4, 8, 16):
        for tuning in ((4, 1, 1, 0, 0), (8, 1, 2, 0, 2)):
            xs = [torch.from_numpy(rng.integers(-127, 128, size=(B, M.cols)).astype(np.int8)).cuda() for M in Ms]
            S = ops.Q8Stack(Ms, batch=B, tuning=tuning + (engine,), xs=xs)
            ys = S.run()
            for W, x, y in zip(Ws, xs, ys):
                assert np.array_equal(y.cpu().numpy(), oracle.matvec_i8(W, x.cpu().numpy())), (W.shape, B, tuning)
    assert ops.device_status() == 0
