"""GPU parity: every kernel through the C ABI against the CPU oracle.

Integer results must be bit-exact: decoded weights equal the reference
encoder's input and y equals the oracle's int64-accumulated int8 matvec.
FP32 outputs are compared with the same fp32 operations done on the host
(y_scaled = float32(y) * scale; requantisation as in
ans-warp-rows-kernel.cu:212-220 and matvansWarpPerRow.cu:62-72), which is exact.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden, cuda_ok
import oracle
from oracle import formats

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import codec, ops, _lib


def rnd_x(rng, B, cols):
    return rng.integers(-127, 128, size=(B, cols)).astype(np.int8)


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


def fp32_scaled(y, s):
    return (y.astype(np.float32) * s.astype(np.float32)[None, :]).astype(np.float32)


@pytest.fixture(autouse=True)
def clean_status():
    ops.device_status(raise_on_error=False)
    yield


# ------------------------------------------------------------------- AWR

def test_awr_cases_all_batches(awr_cases):
    rng = np.random.default_rng(1)
    for name, c in awr_cases.items():
        W = c["W"]
        M = ops.AwrMatrix(c["compressed"], c["offsets"], c["ppf"], c["ppf_cum"], c["ppf_prob"], *W.shape)
        for B in (1, 2, 3, 8, 16, 17):
            x = rnd_x(rng, B, W.shape[1])
            y = M.matvec(torch.from_numpy(x)).cpu().numpy()
            assert np.array_equal(y, oracle.matvec_i8(W, x)), (name, B)
        ops.device_status()


def test_awr_scaled_output(awr_cases):
    c = awr_cases["c1_1024x1024"]
    rng = np.random.default_rng(2)
    s = rng.uniform(1e-3, 1e-2, size=1024).astype(np.float32)
    x = rnd_x(rng, 4, 1024)
    M = ops.AwrMatrix(c["compressed"], c["offsets"], c["ppf"], c["ppf_cum"], c["ppf_prob"], 1024, 1024)
    y, ys = M.matvec(torch.from_numpy(x), scales=s)
    yref = oracle.matvec_i8(c["W"], x)
    assert np.array_equal(y.cpu().numpy(), yref)
    assert np.array_equal(ys.cpu().numpy(), fp32_scaled(yref, s))


def test_awr_chain_requant_and_reference_shim():
    st = formats.read_safetensors(golden("awr_chain.safetensors"))
    raw = np.load(golden("awr_chain_raw.npz"))
    dim = st["initial_vector"].size
    comp = torch.from_numpy(st["compressed"]).cuda()
    v = torch.from_numpy(st["initial_vector"]).cuda()
    v_shim = v.clone()
    for k in range(st["scales"].size):
        args = [torch.from_numpy(np.ascontiguousarray(st[n][k])).cuda()
                for n in ("all_warp_offsets", "all_ppfs", "all_ppfs_cum", "all_ppfs_prob")]
        M = ops.AwrMatrix(st["compressed"], st["all_warp_offsets"][k], st["all_ppfs"][k], st["all_ppfs_cum"][k],
                          st["all_ppfs_prob"][k], dim, dim)
        y = M.matvec(v).cpu().numpy()
        assert np.array_equal(y, oracle.matvec_i8(raw["matrices"][k], v.cpu().numpy()))
        out = M.matvec_requant(v, float(st["scales"][k]))
        # the kernel's fp32 epilogue: rn(float(y) * scale), clamped to int8
        ref8 = np.clip(np.rint(y.astype(np.float32) * np.float32(st["scales"][k])), -128, 127).astype(np.int8)
        assert np.array_equal(out.cpu().numpy(), ref8)
        # the reference launcher signature (buffered/ans-warp-rows.cu:38-60)
        shim_out = torch.empty(dim, dtype=torch.int8, device="cuda")
        ops.mat_vec_mul_coalesced(v_shim, shim_out, dim, dim, float(st["scales"][k]), comp, *args)
        torch.cuda.synchronize()
        assert np.array_equal(shim_out.cpu().numpy(), out.cpu().numpy())
        v, v_shim = out, shim_out
        assert codec.hash_int8_array(v.cpu().numpy()) == int(st["hashes"][k])
    ops.device_status()


def test_awr_full_size_7b_shapes():
    rng = np.random.default_rng(3)
    for shape in ((4096, 4096), (11008, 4096), (4096, 11008)):
        W = gauss(rng, 4.0, shape)
        M = ops.AwrMatrix.encode(W)
        x = rnd_x(rng, 2, shape[1])
        y = M.matvec(torch.from_numpy(x)).cpu().numpy()
        assert np.array_equal(y, oracle.matvec_i8(W, x)), shape
    ops.device_status()


# ------------------------------------------------------------------- WPR

def test_wpr_fixtures_and_chain_hash():
    f = formats.read_wpr_bin(golden("wpr_chain_512.bin"))
    raw = np.load(golden("wpr_chain_512_raw.npz"))
    v = torch.from_numpy(f["vector"]).cuda()
    for k, m in enumerate(f["matrices"]):
        cm = codec.CompressedMatrix(m["rows"], m["cols"], 1.0, m["cursors"], m["min_value"], m["cdf"], m["ppf"],
                                    m["payload"])
        M = ops.WprMatrix(cm)
        y = M.matvec(v)
        yh = y.cpu().numpy()
        assert np.array_equal(yh, oracle.matvec_i8(raw["matrices"][k], v.cpu().numpy()))
        out8, delta = ops.requant_absmax(y)
        d = np.float32(np.float32(np.abs(yh.astype(np.int64)).max()) / np.float32(127))
        assert np.float32(delta.item()) == d
        ref8 = np.rint(yh.astype(np.float32) / d).astype(np.int8)
        assert np.array_equal(out8.cpu().numpy(), ref8)
        v = out8
    # the file's KAT (computed by the script in float64) reproduced by the fp32 GPU chain
    assert codec.hash_int8_array(v.cpu().numpy()) == f["result_hash"]
    ops.device_status()


def test_wpr_plain_method_1024_batches():
    f = formats.read_wpr_bin(golden("wpr_c1_1024.bin"))
    ref = np.load(golden("wpr_c1_1024.npz"))
    m = f["matrices"][0]
    M = ops.WprMatrix(codec.CompressedMatrix(1024, 1024, 1.0, m["cursors"], m["min_value"], m["cdf"], m["ppf"],
                                             m["payload"]))
    y, ys = M.matvec(torch.from_numpy(ref["x"]), scales=ref["scales"])
    assert np.array_equal(y.cpu().numpy(), ref["y"])
    assert np.array_equal(ys.cpu().numpy(), fp32_scaled(ref["y"][None], ref["scales"])[0])
    rng = np.random.default_rng(4)
    for B in (2, 5, 16):
        x = rnd_x(rng, B, 1024)
        assert np.array_equal(M.matvec(torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(ref["W"], x))
    ops.device_status()


def test_wpr_product_encoder_4096():
    rng = np.random.default_rng(5)
    W = gauss(rng, 4.0, (4096, 4096))
    M = ops.WprMatrix.encode(W)
    x = rnd_x(rng, 1, 4096)
    assert np.array_equal(M.matvec(torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(W, x))
    ops.device_status()


# -------------------------------------------------------------------- Q8

Q8_SHAPES = [(64, 512), (45, 301), (33, 7), (1, 100), (100, 1000), (300, 4096)]


@pytest.mark.parametrize("local", [True, False])
@pytest.mark.parametrize("shape", Q8_SHAPES)
def test_q8_small_shapes(shape, local):
    rng = np.random.default_rng(hash(shape) % 1000)
    W = gauss(rng, 3.0, shape)
    M = ops.Q8Matrix.encode(W, local=local)
    assert np.array_equal(M.decode().cpu().numpy(), W)
    for B in (1, 2, 3, 4, 7, 8, 16, 33):
        x = rnd_x(rng, B, shape[1])
        y = M.matvec(torch.from_numpy(x)).cpu().numpy()
        assert np.array_equal(y, oracle.matvec_i8(W, x)), B
    ops.device_status()


@pytest.mark.parametrize("kind", ["const", "all256", "laplace_outliers", "uniform"])
def test_q8_value_distributions(kind):
    rng = np.random.default_rng(9)
    shape = (96, 1536)
    if kind == "const":
        W = np.full(shape, 127, np.int8)
    elif kind == "all256":
        W = rng.permutation(np.tile(np.arange(-128, 128, dtype=np.int8), shape[0] * shape[1] // 256)).reshape(shape)
    elif kind == "laplace_outliers":
        W = np.clip(np.round(rng.laplace(0, 3, shape)), -127, 127).astype(np.int8)
        mask = rng.random(shape) < 0.001
        W[mask] = rng.choice(np.array([-100, 100], np.int8), size=mask.sum())
    else:
        W = rng.integers(-128, 128, size=shape).astype(np.int8)
    for local in (True, False):
        M = ops.Q8Matrix.encode(W, local=local)
        assert np.array_equal(M.decode().cpu().numpy(), W)
        x = rnd_x(rng, 3, shape[1])
        assert np.array_equal(M.matvec(torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(W, x))
    ops.device_status()


@pytest.mark.parametrize("local", [True, False])
def test_q8_full_size_7b_shapes(local):
    rng = np.random.default_rng(6)
    for shape, sigma in (((4096, 4096), 4.0), ((11008, 4096), 2.0), ((4096, 11008), 4.0)):
        W = gauss(rng, sigma, shape)
        M = ops.Q8Matrix.encode(W, local=local)
        s = rng.uniform(1e-3, 1e-2, size=shape[0]).astype(np.float32)
        x = rnd_x(rng, 4, shape[1])
        y, ys = M.matvec(torch.from_numpy(x), scales=s)
        yref = oracle.matvec_i8(W, x)
        assert np.array_equal(y.cpu().numpy(), yref), shape
        assert np.array_equal(ys.cpu().numpy(), fp32_scaled(yref, s)), shape
        # size-independent property: linearity in x
        x2 = rnd_x(rng, 1, shape[1])
        xs = (x[:1].astype(np.int16) + x2.astype(np.int16))
        ok = (np.abs(xs) <= 127).all(axis=0)
        xs = np.where(ok, xs, 0).astype(np.int8)
        x1 = np.where(ok, x[:1], 0).astype(np.int8)
        x2 = np.where(ok, x2, 0).astype(np.int8)
        ya = M.matvec(torch.from_numpy(xs)).cpu().numpy().astype(np.int64)
        yb = M.matvec(torch.from_numpy(x1)).cpu().numpy().astype(np.int64) + \
            M.matvec(torch.from_numpy(x2)).cpu().numpy().astype(np.int64)
        assert np.array_equal(ya, yb)
    ops.device_status()


# ------------------------------------------------------------------ dense

def test_dense_comparator():
    rng = np.random.default_rng(7)
    for shape in ((4096, 4096), (11008, 4096), (4096, 11008), (37, 48)):
        W = gauss(rng, 4.0, shape)
        Wd = torch.from_numpy(W).cuda()
        for B in (1, 4, 16):
            x = rnd_x(rng, B, shape[1])
            assert np.array_equal(ops.dense_matvec(Wd, torch.from_numpy(x)).cpu().numpy(),
                                  oracle.matvec_i8(W, x))
    # 16 vectors x 16384 columns exceed shared memory (passes of 8); 300000 columns exceed it for one
    # vector (x read through the caches)
    for cols in (16384, 300000):
        W = gauss(rng, 2.0, (40, cols))
        Wd = torch.from_numpy(W).cuda()
        for B in (1, 9, 16):
            x = rnd_x(rng, B, cols)
            assert np.array_equal(ops.dense_matvec(Wd, torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(W, x))


# -------------------------------------------------- device-side error paths

def test_q8_corrupt_stream_is_reported_not_faulted():
    rng = np.random.default_rng(8)
    W = gauss(rng, 4.0, (256, 1024))
    enc = codec.q8_encode(W, local=True)
    bad = dict(enc)
    blocks = enc["blocks"].copy()
    blocks[70:70 + 64] ^= np.uint32(0x5A5A5A5A)  # flip bits inside the first block's payload words
    bad["blocks"] = blocks
    M = ops.Q8Matrix(bad)
    M.matvec(torch.from_numpy(rnd_x(rng, 1, 1024)))
    flags = ops.device_status(raise_on_error=False)
    assert flags & _lib.DEV_FINAL_STATE
    # the context is still usable
    good = ops.Q8Matrix(enc)
    x = rnd_x(rng, 1, 1024)
    assert np.array_equal(good.matvec(torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(W, x))
    assert ops.device_status() == 0


def test_q8_offsets_past_buffer_are_rejected_in_kernel():
    rng = np.random.default_rng(10)
    W = gauss(rng, 4.0, (64, 512))
    enc = codec.q8_encode(W, local=False)
    bad = dict(enc)
    off = enc["blk_off"].copy()
    off[-1] = off[-1] + 1000  # last block claims rows beyond the buffer
    bad["blk_off"] = off
    ops.Q8Matrix(bad).matvec(torch.from_numpy(rnd_x(rng, 1, 512)))
    assert ops.device_status(raise_on_error=False) & _lib.DEV_STREAM_OVERRUN


def test_awr_offsets_past_buffer_are_reported():
    rng = np.random.default_rng(12)
    W = gauss(rng, 4.0, (32, 256))
    comp, offs, mn, cdf = codec.compress_ans_warp_rows(W)
    p, pc, pp = codec.decoder_model_from_128bit_encoder_model(mn, cdf)
    offs = offs.copy()
    offs[5] = comp.size // 4 + 64  # beyond the stream
    M = ops.AwrMatrix(comp, offs, codec.pack_4bytes(p), codec.pack_4bytes(pc), codec.pack_4bytes(pp), 32, 256)
    M.matvec(torch.from_numpy(rnd_x(rng, 1, 256)))
    assert ops.device_status(raise_on_error=False) & _lib.DEV_STREAM_OVERRUN


def test_wpr_corrupt_payload_is_reported():
    f = formats.read_wpr_bin(golden("wpr_c1_1024.bin"))
    m = f["matrices"][0]
    pay = m["payload"].copy()
    pay[300:900] ^= np.uint16(0x3C3C)
    M = ops.WprMatrix(codec.CompressedMatrix(1024, 1024, 1.0, m["cursors"], m["min_value"], m["cdf"], m["ppf"], pay))
    M.matvec(torch.from_numpy(f["vector"]))
    assert ops.device_status(raise_on_error=False) & _lib.DEV_FINAL_STATE


def test_wpr_cursors_past_payload_are_reported():
    # a row whose cursor points past the payload (or near 2^32) reads zeros and raises the overrun flag
    f = formats.read_wpr_bin(golden("wpr_c1_1024.bin"))
    m = f["matrices"][0]
    for bad in (m["payload"].size + 5, 0xFFFFFF00):
        cur = m["cursors"].copy()
        cur[7] = bad
        M = ops.WprMatrix(codec.CompressedMatrix(1024, 1024, 1.0, cur, m["min_value"], m["cdf"], m["ppf"],
                                                 m["payload"]))
        M.matvec(torch.from_numpy(f["vector"]))
        assert ops.device_status(raise_on_error=False) & _lib.DEV_STREAM_OVERRUN


def test_bounded_wait_times_out_with_status():
    rng = np.random.default_rng(13)
    W = gauss(rng, 4.0, (64, 512))
    M = ops.Q8Matrix.encode(W)
    L = _lib.lib()
    try:
        _lib.check(L.mv_debug_inject(1, 2000))  # MV_INJECT_WAIT_LIMIT
        _lib.check(L.mv_debug_inject(2, 1))     # MV_INJECT_DROP_COPY
        M.matvec(torch.from_numpy(rnd_x(rng, 1, 512)))
        flags = ops.device_status(raise_on_error=False)
    finally:
        L.mv_debug_inject(2, 0)
        L.mv_debug_inject(1, 0)
    assert flags & _lib.DEV_WAIT_TIMEOUT
    x = rnd_x(rng, 1, 512)
    assert np.array_equal(M.matvec(torch.from_numpy(x)).cpu().numpy(), oracle.matvec_i8(W, x))
    assert ops.device_status() == 0
