"""The reference's "ans-warp-stripes" layout on the GPU (mv_aws_matvec,
mv_aws_matvec_requant, the renamed reference launcher), bit-exact against the
oracle and the reference's own fixtures and chain hashes."""
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


def cases():
    z = np.load(golden("aws_cases.npz"))
    names = sorted({k[:-2] for k in z.files if k.endswith("_W")})
    return {n: {k[len(n) + 1:]: z[k] for k in z.files if k.startswith(n + "_")} for n in names}


def fp32_scaled(y, s):
    return (y.astype(np.float32) * s[None, :].astype(np.float32)).astype(np.float32)


@pytest.mark.parametrize("B", [1, 3, 16, 20])
def test_stripes_reference_fixtures(B):
    rng = np.random.default_rng(B)
    for name, c in cases().items():
        W = c["W"]
        rows, cols = W.shape
        M = ops.AwsMatrix(c["compressed"], c["offsets"], c["ppf"], c["ppf_cum"], c["ppf_prob"], rows, cols)
        x = rng.integers(-127, 128, size=(B, cols)).astype(np.int8)
        s = rng.uniform(1e-3, 1e-2, size=rows).astype(np.float32)
        y, ys = M.matvec(torch.from_numpy(x), scales=s)
        yref = oracle.matvec_i8(W, x)
        assert np.array_equal(y.cpu().numpy(), yref), name
        assert np.array_equal(ys.cpu().numpy(), fp32_scaled(yref, s)), name
    assert ops.device_status() == 0


def test_stripes_chain_requant_shim_and_reference_hashes():
    st = formats.read_safetensors(golden("aws_chain.safetensors"))
    dim = st["initial_vector"].size
    comp = torch.from_numpy(st["compressed"]).cuda()
    v = torch.from_numpy(st["initial_vector"]).cuda()
    v_shim = v.clone()
    for k in range(st["scales"].size):
        M = ops.AwsMatrix(st["compressed"], st["all_warp_offsets"][k], st["all_ppfs"][k], st["all_ppfs_cum"][k],
                          st["all_ppfs_prob"][k], dim, dim)
        y = M.matvec(v).cpu().numpy()
        out = M.matvec_requant(v, float(st["scales"][k]))
        ref8 = np.clip(np.rint(y.astype(np.float32) * np.float32(st["scales"][k])), -128, 127).astype(np.int8)
        assert np.array_equal(out.cpu().numpy(), ref8)
        args = [torch.from_numpy(np.ascontiguousarray(st[n][k])).cuda()
                for n in ("all_warp_offsets", "all_ppfs", "all_ppfs_cum", "all_ppfs_prob")]
        shim_out = torch.empty(dim, dtype=torch.int8, device="cuda")
        ops.mat_vec_mul_coalesced_stripes(v_shim, shim_out, dim, dim, float(st["scales"][k]), comp, *args)
        torch.cuda.synchronize()
        assert np.array_equal(shim_out.cpu().numpy(), out.cpu().numpy())
        v, v_shim = out, shim_out
        assert codec.hash_int8_array(v.cpu().numpy()) == int(st["hashes"][k]), k
    assert ops.device_status() == 0


def test_stripes_full_size_7b_shapes():
    rng = np.random.default_rng(5)
    for shape in ((4096, 4096), (11008, 4096), (4096, 11008)):
        W = np.clip(np.round(rng.normal(0, 4.0, size=shape)), -127, 127).astype(np.int8)
        M = ops.AwsMatrix.encode(W)
        x = rng.integers(-127, 128, size=(2, shape[1])).astype(np.int8)
        assert np.array_equal(M.matvec(torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(W, x)), shape
    assert ops.device_status() == 0


def test_stripes_rejects_bad_shapes():
    c = cases()["s4_64x512"]
    M = ops.AwsMatrix(c["compressed"], c["offsets"], c["ppf"], c["ppf_cum"], c["ppf_prob"], 48, 512)
    with pytest.raises(_lib.MatvansError):
        M.matvec(torch.zeros((1, 512), dtype=torch.int8))
