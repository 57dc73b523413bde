"""The product's C++ encoders and file readers against the reference's outputs.

The fixtures were written by the reference's own Python encoders
(tests/golden/gen_golden.py); every stream the product encoder writes for the
same matrix must be byte-identical (WPR padding words are zero in both).
"""
import os

import numpy as np
import pytest

from conftest import golden
from oracle import formats
import oracle
from matvans_b200 import codec


def test_awr_encoder_byte_identical_on_cases(awr_cases):
    for name, c in awr_cases.items():
        comp, offs, mn, cdf = codec.compress_ans_warp_rows(c["W"], 32)
        assert np.array_equal(comp, c["compressed"]), name
        assert np.array_equal(offs, c["offsets"]), name
        assert mn == int(c["min"][0]), name
        assert np.array_equal(cdf, c["cdf"]), name
        p, pc, pp = codec.decoder_model_from_128bit_encoder_model(mn, cdf)
        assert np.array_equal(codec.pack_4bytes(p), c["ppf"]), name
        assert np.array_equal(codec.pack_4bytes(pc), c["ppf_cum"]), name
        assert np.array_equal(codec.pack_4bytes(pp), c["ppf_prob"]), name


def test_awr_model_mirror(awr_cases):
    for name, c in awr_cases.items():
        _, _, mn, cdf = codec.fit_128bit_encoder_model(c["W"])
        assert mn == int(c["min"][0]) and np.array_equal(cdf, c["cdf"]), name


def test_compress_all_matrices_reproduces_reference_file(tmp_path):
    raw = np.load(golden("awr_chain_raw.npz"))
    out = tmp_path / "chain.safetensors"
    codec.compress_all_matrices(raw["matrices"], raw["initial_vector"], raw["scales"], raw["hashes"],
                                codec.compress_ans_warp_rows, str(out))
    mine = formats.read_safetensors(str(out))
    ref = formats.read_safetensors(golden("awr_chain.safetensors"))
    assert sorted(mine) == sorted(ref)
    for k in ref:
        assert mine[k].dtype == ref[k].dtype and np.array_equal(mine[k], ref[k]), k


def test_cpp_safetensors_reader_matches_plain_reader(tmp_path):
    ref = formats.read_safetensors(golden("awr_chain.safetensors"))
    mine = codec.load_safetensors(golden("awr_chain.safetensors"))
    assert sorted(mine) == sorted(ref)
    for k in ref:
        assert mine[k].dtype == ref[k].dtype and mine[k].shape == ref[k].shape and np.array_equal(mine[k], ref[k])


@pytest.mark.parametrize("damage", ["truncate", "header_len", "offsets"])
def test_cpp_safetensors_reader_rejects_damaged_files(tmp_path, damage):
    blob = bytearray(open(golden("awr_chain.safetensors"), "rb").read())
    if damage == "truncate":
        blob = blob[:len(blob) // 2]
    elif damage == "header_len":
        blob[0:8] = (len(blob) * 2).to_bytes(8, "little")
    else:
        i = blob.index(b'"data_offsets":[')
        blob[i + 16:i + 17] = b"9"
    p = tmp_path / "bad.safetensors"
    p.write_bytes(bytes(blob))
    with pytest.raises(Exception):
        codec.load_safetensors(str(p))


def test_wpr_encoder_byte_identical():
    for binf, rawf, key in (("wpr_chain_512.bin", "wpr_chain_512_raw.npz", "matrices"),
                            ("wpr_c1_1024.bin", "wpr_c1_1024.npz", "W")):
        f = formats.read_wpr_bin(golden(binf))
        raw = np.load(golden(rawf))
        mats = raw[key] if raw[key].ndim == 3 else raw[key][None]
        for m, W in zip(f["matrices"], mats):
            cm = codec.encode_matrix(W)
            assert cm.min_value == m["min_value"]
            assert np.array_equal(cm.cdf, m["cdf"])
            assert np.array_equal(cm.ppf, m["ppf"])
            assert np.array_equal(cm.cursors, m["cursors"])
            assert np.array_equal(cm.payload, m["payload"])


def test_wpr_model_mirror():
    f = formats.read_wpr_bin(golden("wpr_c1_1024.bin"))
    W = np.load(golden("wpr_c1_1024.npz"))["W"]
    mn, grid, cdf, H, CE = codec.create_entropy_model(W, 8)
    assert mn == f["matrices"][0]["min_value"]
    assert np.array_equal((cdf & 0xFF).astype(np.uint8), f["matrices"][0]["cdf"])
    assert np.array_equal(codec.create_ppf(cdf), f["matrices"][0]["ppf"])
    assert 4.0 < H < CE < 4.2


def test_wpr_bin_write_read_round_trip(tmp_path):
    f = formats.read_wpr_bin(golden("wpr_chain_512.bin"))
    hdr, vec, mats = codec.read_wpr_bin(golden("wpr_chain_512.bin"))
    assert hdr["num_matrices"] == 3 and hdr["result_hash"] == f["result_hash"]
    assert np.array_equal(vec, f["vector"])
    out = tmp_path / "rt.bin"
    codec.write_wpr_bin(str(out), mats, vec, hdr["result_hash"])
    assert out.read_bytes() == open(golden("wpr_chain_512.bin"), "rb").read()


def test_wpr_bin_reader_rejects_truncation(tmp_path):
    blob = open(golden("wpr_c1_1024.bin"), "rb").read()
    p = tmp_path / "t.bin"
    p.write_bytes(blob[: len(blob) - 1000])
    with pytest.raises(Exception):
        codec.read_wpr_bin(str(p))


def test_hash_matches_oracle():
    rng = np.random.default_rng(3)
    v = rng.integers(-128, 128, size=4097).astype(np.int8)
    assert codec.hash_int8_array(v) == oracle.hash_int8(v)


def test_shape_errors():
    from matvans_b200 import MatvansError
    with pytest.raises(MatvansError):
        codec.compress_ans_warp_rows(np.zeros((4, 100), np.int8))
    with pytest.raises(MatvansError):
        codec.encode_matrix(np.zeros((4, 1000), np.int8))
    wide = np.arange(-128, 128, dtype=np.int8).repeat(2).reshape(2, 256)
    with pytest.raises(MatvansError):
        codec.compress_ans_warp_rows(wide)


def test_aws_encoder_byte_identical_on_cases():
    z = np.load(golden("aws_cases.npz"))
    names = sorted({k[:-2] for k in z.files if k.endswith("_W")})
    assert len(names) >= 8
    for name in names:
        comp, offs, mn, cdf = codec.compress_ans_warp_stripes(z[name + "_W"], 32)
        assert np.array_equal(comp, z[name + "_compressed"]), name
        assert np.array_equal(offs, z[name + "_offsets"]), name
        assert mn == int(z[name + "_min"][0]) and np.array_equal(cdf, z[name + "_cdf"]), name


def test_compress_all_matrices_stripes_reproduces_reference_file(tmp_path):
    raw = np.load(golden("awr_chain_raw.npz"))
    out = tmp_path / "chain_stripes.safetensors"
    codec.compress_all_matrices(raw["matrices"], raw["initial_vector"], raw["scales"], raw["hashes"],
                                codec.compress_ans_warp_stripes, str(out))
    mine = formats.read_safetensors(str(out))
    ref = formats.read_safetensors(golden("aws_chain.safetensors"))
    assert sorted(mine) == sorted(ref)
    for k in ref:
        assert mine[k].dtype == ref[k].dtype and np.array_equal(mine[k], ref[k]), k


def test_aws_encoder_rejects_bad_shapes():
    with pytest.raises(Exception):
        codec.compress_ans_warp_stripes(np.zeros((48, 128), np.int8))
    with pytest.raises(Exception):
        codec.compress_ans_warp_stripes(np.zeros((32, 130), np.int8))
