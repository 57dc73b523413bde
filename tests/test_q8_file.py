"""The Q8 layout's file form (mv_q8_save / mv_q8_file_* / mv_q8_load): a safetensors file in the reference's
convention (buffered/encoder.py:473-511).  CPU: round trip of several matrices with row scales and chain
data, and rejection of damaged files.  GPU: a file loaded through the C ABI (device upload) and through the
Python loader decodes to the exact product the oracle computes."""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import cuda_ok
from matvans_b200 import _lib, codec


def _mats(rng):
    shapes = [(64, 256, 4.0, True), (33, 160, 2.0, False), (96, 512, 6.0, True)]
    out = []
    for r, c, s, local in shapes:
        W = np.clip(np.round(rng.normal(0, s, size=(r, c))), -127, 127).astype(np.int8)
        out.append((W, codec.q8_encode(W, local=local)))
    return out


def test_q8_file_round_trip(tmp_path):
    rng = np.random.default_rng(41)
    mats = _mats(rng)
    encs = [e for _, e in mats]
    scales = [rng.uniform(1e-3, 1e-2, e["rows"]).astype(np.float32) if i != 1 else None
              for i, e in enumerate(encs)]
    chain = {"initial_vector": rng.integers(-127, 128, 256).astype(np.int8),
             "scales": np.array([0.5, 0.25, 0.125], np.float32), "hashes": np.array([1, 2, 3], np.uint32)}
    p = tmp_path / "m.safetensors"
    codec.save_q8(p, encs, row_scales=scales, chain=chain)
    got, got_scales, got_chain = codec.load_q8(p)
    assert len(got) == 3
    for e, g in zip(encs, got):
        for k in ("blocks", "blk_off", "tbl", "tbl_off"):
            assert np.array_equal(np.asarray(e[k]).view(g[k].dtype), g[k]), k
        for k in ("rows", "cols", "seg_quads", "nseg", "local", "max_blk_rows", "tbl_stripe_max", "payload_bytes"):
            assert int(e[k]) == int(g[k]), k
    assert got_scales[1] is None
    assert np.array_equal(got_scales[0], scales[0]) and np.array_equal(got_scales[2], scales[2])
    for k in chain:
        assert np.array_equal(got_chain[k], chain[k]), k
    # the tensor names follow the reference file's convention
    names = set(codec.load_safetensors(p))
    assert {"q8_meta", "q8_blocks", "q8_blocks_start", "initial_vector", "scales", "hashes"} <= names


def test_q8_file_without_chain(tmp_path):
    rng = np.random.default_rng(42)
    (W, e), = _mats(rng)[:1]
    p = tmp_path / "one.safetensors"
    codec.save_q8(p, [e])
    got, sc, chain = codec.load_q8(p)
    assert len(got) == 1 and sc == [None] and all(v is None for v in chain.values())


def test_q8_file_rejects_damage(tmp_path):
    rng = np.random.default_rng(43)
    mats = _mats(rng)
    p = tmp_path / "m.safetensors"
    codec.save_q8(p, [e for _, e in mats])
    t = codec.load_safetensors(p)
    # a block offset beyond the block data
    bad = dict(t)
    bo = bad["q8_blk_off"].copy()
    bo[int(bad["q8_blk_off_start"][1]) - 1] = 10 ** 6
    bad["q8_blk_off"] = bo
    codec.save_safetensors(tmp_path / "bad1.safetensors", bad)
    with pytest.raises(_lib.MatvansError):
        codec.load_q8(tmp_path / "bad1.safetensors")
    # nseg inconsistent with cols and seg_quads
    bad = dict(t)
    meta = bad["q8_meta"].copy()
    meta[0, 3] += 1
    bad["q8_meta"] = meta
    codec.save_safetensors(tmp_path / "bad2.safetensors", bad)
    with pytest.raises(_lib.MatvansError):
        codec.load_q8(tmp_path / "bad2.safetensors")
    # start offsets past the concatenated array
    bad = dict(t)
    st = bad["q8_tbl_start"].copy()
    st[-1] += 100
    bad["q8_tbl_start"] = st
    codec.save_safetensors(tmp_path / "bad3.safetensors", bad)
    with pytest.raises(_lib.MatvansError):
        codec.load_q8(tmp_path / "bad3.safetensors")
    # truncated file
    raw = open(p, "rb").read()
    (tmp_path / "trunc.safetensors").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(_lib.MatvansError):
        codec.load_q8(tmp_path / "trunc.safetensors")
    # not a Q8 file
    codec.save_safetensors(tmp_path / "other.safetensors", {"x": np.zeros(4, np.int8)})
    with pytest.raises(_lib.MatvansError):
        codec.load_q8(tmp_path / "other.safetensors")


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")
def test_q8_file_loads_to_exact_products_on_gpu(tmp_path):
    import torch
    from matvans_b200 import ops
    rng = np.random.default_rng(44)
    mats = _mats(rng)
    p = tmp_path / "m.safetensors"
    codec.save_q8(p, [e for _, e in mats])
    L = _lib.lib()
    for i, (W, _) in enumerate(mats):
        x = rng.integers(-127, 128, size=(3, W.shape[1])).astype(np.int8)
        ref = oracle.matvec_i8(W, x)
        # C ABI: read, check and upload in one call
        h = ctypes.c_void_p()
        _lib.check(L.mv_q8_load(str(p).encode(), i, ctypes.byref(h)))
        try:
            view = L.mv_q8_matrix_view(h)
            xd = torch.from_numpy(x).cuda()
            y = torch.empty((3, W.shape[0]), dtype=torch.int32, device="cuda")
            _lib.check(L.mv_q8_matvec(view, ctypes.c_void_p(xd.data_ptr()), 3, ctypes.c_void_p(y.data_ptr()), None,
                                      None, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
            torch.cuda.synchronize()
            assert np.array_equal(y.cpu().numpy(), ref), f"matrix {i} via mv_q8_load"
        finally:
            L.mv_q8_matrix_free(h)
    # Python loader into one persistent launch
    Ms, _, _ = ops.load_q8(p)
    xs = [torch.from_numpy(rng.integers(-127, 128, size=(2, M.cols)).astype(np.int8)).cuda() for M in Ms]
    S = ops.Q8Stack(Ms, batch=2, xs=xs)
    S.run()
    torch.cuda.synchronize()
    for (W, _), x, y in zip(mats, xs, S.ys):
        assert np.array_equal(y.cpu().numpy(), oracle.matvec_i8(W, x.cpu().numpy()))
    ops.device_status()
