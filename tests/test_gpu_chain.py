"""Chained pipeline in one persistent, cooperative launch (mv_q8_chain_matvec):
y_j = W_j x_j, x_{j+1} = clamp(round_half_even(fp32(y_j) * scale_j), -128, 127),
the reference's end-to-end workload of buffered/ans-warp-rows.cu:208-221.
Pinned by the reference's own chain: the hashes its encoder script stored for
every step of the seed-20250829 pipeline are reproduced from the same matrices
re-encoded in the Q8-stripe layout."""
import numpy as np
import pytest

from conftest import cuda_ok, golden
import oracle
from oracle import formats

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import codec, ops, _lib


@pytest.fixture(autouse=True)
def clean_status():
    ops.device_status(raise_on_error=False)
    yield


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


def busy_scales(Ws, x, target=40.0):
    """Per-matrix scales that keep the int8 activations of the chain around +-target."""
    scales = []
    for W in Ws:
        y = oracle.matvec_i8(W, x)
        s = float(np.float32(target / max(1.0, float(y.astype(np.float64).std()))))
        scales.append(s)
        x = np.clip(np.rint(y.astype(np.float32) * np.float32(s)), -128, 127).astype(np.int8)
    return scales


def host_chain(Ws, scales, x):
    """The reference semantics on the host: int64 matvec, fp32 product, round half to even, clamp."""
    xs = [x]
    for W, s in zip(Ws, scales):
        y = oracle.matvec_i8(W, xs[-1])
        xs.append(np.clip(np.rint(y.astype(np.float32) * np.float32(s)), -128, 127).astype(np.int8))
    return xs


@pytest.mark.parametrize("local", [True, False])
def test_chain_reproduces_reference_hashes(local):
    st = formats.read_safetensors(golden("awr_chain.safetensors"))
    raw = np.load(golden("awr_chain_raw.npz"))
    Ws = [raw["matrices"][k] for k in range(st["scales"].size)]
    Ms = [ops.Q8Matrix.encode(W, local=local) for W in Ws]
    x0 = torch.from_numpy(st["initial_vector"].reshape(1, -1)).cuda()
    C = ops.Q8Chain(Ms, [float(s) for s in st["scales"]], batch=1, x0=x0)
    for _ in range(2):  # the counters are reset by every call
        C.run()
        torch.cuda.synchronize()
        outs = [C.xs[k + 1] for k in range(len(Ms) - 1)] + [C.out8]
        for k, v in enumerate(outs):
            assert codec.hash_int8_array(v.cpu().numpy().reshape(-1)) == int(st["hashes"][k]), k
    assert ops.device_status() == 0


@pytest.mark.parametrize("B", [1, 3, 8, 16])
@pytest.mark.parametrize("tuning", [(4, 1, 1, 0), (8, 2, 2, 0), (1, 1, 1, 0), (8, 1, 1, 0, 0, 1), None])
def test_chain_random(B, tuning):
    rng = np.random.default_rng(B * 7 + (tuning or (0,))[0])
    dims = [512, 1008, 256, 4096, 512]
    Ws = [gauss(rng, rng.uniform(2, 6), (dims[i + 1], dims[i])) for i in range(len(dims) - 1)]
    Ms = [ops.Q8Matrix.encode(W, local=(i % 2 == 0)) for i, W in enumerate(Ws)]
    x = rng.integers(-127, 128, size=(B, dims[0])).astype(np.int8)
    scales = busy_scales(Ws, x)
    C = ops.Q8Chain(Ms, scales, batch=B, tuning=tuning, x0=torch.from_numpy(x).cuda())
    C.run()
    ref = host_chain(Ws, scales, x)
    for j in range(len(Ms)):
        assert np.array_equal(C.ys[j].cpu().numpy(), oracle.matvec_i8(Ws[j], ref[j])), j
        got = C.xs[j + 1] if j + 1 < len(Ms) else C.out8
        assert np.array_equal(got.cpu().numpy(), ref[j + 1]), j
    assert np.abs(ref[-1].astype(int)).max() > 10  # the chain did not collapse to zeros
    assert ops.device_status() == 0


def test_chain_7b_shapes():
    rng = np.random.default_rng(77)
    shapes = [(4096, 4096), (11008, 4096), (4096, 11008)]
    Ws = [gauss(rng, 4.0, sh) for sh in shapes]
    Ms = [ops.Q8Matrix.encode(W, local=True) for W in Ws]
    for B in (1, 16):
        x = rng.integers(-127, 128, size=(B, 4096)).astype(np.int8)
        scales = busy_scales(Ws, x)
        C = ops.Q8Chain(Ms, scales, batch=B, x0=torch.from_numpy(x).cuda())
        C.run()
        ref = host_chain(Ws, scales, x)
        assert np.array_equal(C.out8.cpu().numpy(), ref[-1])
        assert np.array_equal(C.xs[1].cpu().numpy(), ref[1])
    assert ops.device_status() == 0


def test_chain_rejects_mismatched_shapes():
    Ms = [ops.Q8Matrix.encode(np.ones((64, 128), np.int8)), ops.Q8Matrix.encode(np.ones((64, 128), np.int8))]
    with pytest.raises(_lib.MatvansError):
        ops.Q8Chain(Ms, [1.0, 1.0])
