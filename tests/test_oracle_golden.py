"""Pin the CPU oracle against the fixtures made by the reference's own encoders.

Every fixture under tests/golden/ was produced by buffered/encoder.py or
matvansWarpPerRow/create_matrices_WarpPerRow.py (tests/golden/gen_golden.py).
Coding is lossless, so the oracle must decode each stream back to the exact
int8 matrix the reference encoded, and the reference's stored hashes of the
requantised chain (its only known-answer test, ans-warp-rows.cu:102-118 and
matvansWarpPerRow.cu:355-367) must be reproduced from the oracle's int32 y.
"""
import numpy as np
import pytest

import oracle
from oracle import formats
from conftest import golden


def test_hash_matches_reference_definition():
    # buffered/encoder.py:8-20, restated in Python for this check only
    v = np.arange(-128, 128, dtype=np.int8)
    h = 0
    for b in v.astype(np.uint8):
        h = ((h >> 27) | (h << 5)) & 0xFFFFFFFF
        h = ((h ^ int(b)) * 0x27220A95) & 0xFFFFFFFF
    assert oracle.hash_int8(v) == h
    assert oracle.hash_int8(np.zeros(0, np.int8)) == 0


def test_matvec_int64_accumulation():
    rng = np.random.default_rng(0)
    W = rng.integers(-128, 128, size=(17, 300)).astype(np.int8)
    x = rng.integers(-128, 128, size=(3, 300)).astype(np.int8)
    ref = (W.astype(np.int64) @ x.astype(np.int64).T).T
    assert np.array_equal(oracle.matvec_i8(W, x), ref)


def test_awr_chain_decodes_and_reproduces_reference_hashes():
    st = formats.read_safetensors(golden("awr_chain.safetensors"))
    raw = np.load(golden("awr_chain_raw.npz"))
    mats = raw["matrices"]
    count, dim = mats.shape[0], mats.shape[1]
    assert st["all_warp_offsets"].shape == (count, dim)
    v = st["initial_vector"]
    assert np.array_equal(v, raw["initial_vector"])
    for k in range(count):
        W = oracle.awr_decode(st["compressed"], st["all_warp_offsets"][k], dim, dim,
                              st["all_ppfs"][k], st["all_ppfs_cum"][k], st["all_ppfs_prob"][k])
        assert np.array_equal(W, mats[k]), f"matrix {k} does not round-trip"
        y = oracle.awr_matvec(st["compressed"], st["all_warp_offsets"][k], dim, dim,
                              st["all_ppfs"][k], st["all_ppfs_cum"][k], st["all_ppfs_prob"][k], v,
                              nthreads=4)
        assert np.array_equal(y, oracle.matvec_i8(mats[k], v))
        # the reference's own requantisation, buffered/encoder.py:46-51 (NumPy 2:
        # int32 * float32 promotes to float64, then round-half-even)
        v = np.round(y * st["scales"][k]).astype(np.int8)
        assert oracle.hash_int8(v) == int(st["hashes"][k]), f"hash of step {k}"


def test_awr_cases_round_trip(awr_cases):
    for name, c in awr_cases.items():
        W = c["W"]
        rows, cols = W.shape
        got = oracle.awr_decode(c["compressed"], c["offsets"], rows, cols, c["ppf"], c["ppf_cum"],
                                c["ppf_prob"])
        assert np.array_equal(got, W), name
        rng = np.random.default_rng(7)
        x = rng.integers(-127, 128, size=(2, cols)).astype(np.int8)
        y = oracle.awr_matvec(c["compressed"], c["offsets"], rows, cols, c["ppf"], c["ppf_cum"],
                              c["ppf_prob"], x, nthreads=3)
        assert np.array_equal(y, oracle.matvec_i8(W, x)), name


def test_awr_rejects_bad_shape(awr_cases):
    c = awr_cases["s4_64x512"]
    with pytest.raises(oracle.OracleError):
        oracle.awr_decode(c["compressed"], c["offsets"], 64, 500, c["ppf"], c["ppf_cum"], c["ppf_prob"])


def test_wpr_chain_decodes_and_reproduces_reference_hash():
    f = formats.read_wpr_bin(golden("wpr_chain_512.bin"))
    raw = np.load(golden("wpr_chain_512_raw.npz"))
    assert np.array_equal(f["vector"], raw["vector"])
    v = f["vector"]
    v_delta = 1.0
    for k, m in enumerate(f["matrices"]):
        W = oracle.wpr_decode(m["payload"], m["cursors"], m["rows"], m["cols"], m["min_value"],
                              m["cdf"], m["ppf"])
        assert np.array_equal(W, raw["matrices"][k]), f"matrix {k} does not round-trip"
        y = oracle.wpr_matvec(m["payload"], m["cursors"], m["rows"], m["cols"], m["min_value"],
                              m["cdf"], m["ppf"], v, nthreads=2)
        assert np.array_equal(y, oracle.matvec_i8(W, v))
        # the script's float64 chain, create_matrices_WarpPerRow.py:72-87
        v_f = y.astype(float) * raw["w_deltas"][k] * v_delta
        v_delta = np.abs(v_f).max() / 127
        v = np.round(v_f / v_delta).astype(np.int8)
    assert oracle.hash_int8(v) == f["result_hash"] == int(raw["result_hash"][0])


def test_wpr_plain_method_1024():
    f = formats.read_wpr_bin(golden("wpr_c1_1024.bin"))
    ref = np.load(golden("wpr_c1_1024.npz"))
    m = f["matrices"][0]
    assert (m["rows"], m["cols"]) == (1024, 1024)
    W = oracle.wpr_decode(m["payload"], m["cursors"], 1024, 1024, m["min_value"], m["cdf"], m["ppf"])
    assert np.array_equal(W, ref["W"])
    y = oracle.wpr_matvec(m["payload"], m["cursors"], 1024, 1024, m["min_value"], m["cdf"], m["ppf"],
                          ref["x"], nthreads=4)
    assert np.array_equal(y, ref["y"])
    assert np.array_equal(f["vector"], ref["x"])


# ------------------------------------------------------------ ans-warp-stripes

def _aws_cases():
    z = np.load(golden("aws_cases.npz"))
    names = sorted({k[:-2] for k in z.files if k.endswith("_W")})
    return {n: {k[len(n) + 1:]: z[k] for k in z.files if k.startswith(n + "_")} for n in names}


def test_aws_cases_round_trip():
    for name, c in _aws_cases().items():
        W = c["W"]
        rows, cols = W.shape
        got = oracle.aws_decode(c["compressed"], c["offsets"], rows, cols, c["ppf"], c["ppf_cum"], c["ppf_prob"])
        assert np.array_equal(got, W), name
        x = np.random.default_rng(8).integers(-127, 128, size=(3, cols)).astype(np.int8)
        y = oracle.aws_matvec(c["compressed"], c["offsets"], rows, cols, c["ppf"], c["ppf_cum"], c["ppf_prob"], x)
        assert np.array_equal(y, oracle.matvec_i8(W, x)), name


def test_aws_chain_decodes_and_reproduces_reference_hashes():
    # the reference's seed-20250829 pipeline compressed with compress_ans_warp_stripes: same matrices and
    # hashes as the rows-layout chain
    st = formats.read_safetensors(golden("aws_chain.safetensors"))
    raw = np.load(golden("awr_chain_raw.npz"))
    mats = raw["matrices"]
    count, dim = mats.shape[0], mats.shape[1]
    assert st["all_warp_offsets"].shape == (count, dim // 32)
    v = st["initial_vector"]
    for k in range(count):
        W = oracle.aws_decode(st["compressed"], st["all_warp_offsets"][k], dim, dim,
                              st["all_ppfs"][k], st["all_ppfs_cum"][k], st["all_ppfs_prob"][k])
        assert np.array_equal(W, mats[k]), f"matrix {k} does not round-trip"
        y = oracle.aws_matvec(st["compressed"], st["all_warp_offsets"][k], dim, dim,
                              st["all_ppfs"][k], st["all_ppfs_cum"][k], st["all_ppfs_prob"][k], v)
        v = np.round(y * st["scales"][k]).astype(np.int8)  # the reference's requantisation, encoder.py:46-51
        assert oracle.hash_int8(v) == int(st["hashes"][k]), k


def test_aws_rejects_bad_shape():
    c = _aws_cases()["s4_64x512"]
    with pytest.raises(oracle.OracleError):
        oracle.aws_decode(c["compressed"], c["offsets"], 48, 512, c["ppf"], c["ppf_cum"], c["ppf_prob"])


def test_oracle_awr_encoder_matches_reference_encoder(awr_cases):
    """The oracle's C restatement of the reference encoder (used by the benchmark's CPU legs, which must not
    load the product library) is byte-identical to buffered/encoder.py on every reference-made fixture."""
    for name, c in awr_cases.items():
        comp, offs, ppf, cum, prob = oracle.awr_encode(c["W"])
        assert np.array_equal(comp, c["compressed"]), name
        assert np.array_equal(offs, c["offsets"]), name
        for got, key in ((ppf, "ppf"), (cum, "ppf_cum"), (prob, "ppf_prob")):
            assert np.array_equal(got, c[key]), (name, key)


def test_oracle_awr_encoder_rejects_unencodable():
    with pytest.raises(oracle.OracleError):
        oracle.awr_encode(np.zeros((2, 100), np.int8))  # cols % 128 != 0 (encoder.py:397)
    with pytest.raises(oracle.OracleError):
        oracle.awr_encode(np.arange(-128, 128, dtype=np.int8).reshape(2, 128))  # > 128 distinct values
