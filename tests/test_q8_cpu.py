"""Q8-stripe encoder checks on the CPU: lossless round trip through a plain
Python decoder, table invariants, edge shapes and value distributions."""
import numpy as np
import pytest

from matvans_b200 import codec
import q8_py


def gauss(rng, s, shape):
    return np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)


CASES = {
    "s4_64x512_local": (lambda r: gauss(r, 4, (64, 512)), True, 0),
    "s4_64x512_global": (lambda r: gauss(r, 4, (64, 512)), False, 0),
    "s2_ragged_45x301": (lambda r: gauss(r, 2, (45, 301)), True, 0),
    "s1_ragged_33x7": (lambda r: gauss(r, 1, (33, 7)), False, 0),
    "const_40x130": (lambda r: np.full((40, 130), -128, np.int8), True, 0),
    "const127_32x64": (lambda r: np.full((32, 64), 127, np.int8), False, 0),
    "all256_32x512": (lambda r: r.permutation(np.tile(np.arange(-128, 128, dtype=np.int8), 64)).reshape(32, 512),
                      True, 0),
    "uniform_8bit_32x256": (lambda r: r.integers(-128, 128, size=(32, 256)).astype(np.int8), False, 16),
    "laplace_outliers_64x384": (lambda r: np.where(r.random((64, 384)) < 0.001,
                                                   r.choice([-100, 100], size=(64, 384)),
                                                   np.clip(np.round(r.laplace(0, 3, (64, 384))), -127, 127)
                                                   ).astype(np.int8), True, 0),
    "one_row_1x100": (lambda r: gauss(r, 4, (1, 100)), True, 5),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_q8_round_trip(name):
    gen, local, sq = CASES[name]
    W = gen(np.random.default_rng(11))
    enc = codec.q8_encode(W, local=local, seg_quads=sq)
    assert np.array_equal(q8_py.decode(enc), W)
    # tables: freqs in 1..255 summing to 256, symbols sorted and unique
    t, off = enc["tbl"], enc["tbl_off"]
    for i in range(len(off) - 1):
        e = t[off[i]:off[i + 1]]
        f = e >> 8
        assert f.min() >= 1 and f.max() <= 255 and f.sum() == 256
        s = e & 0xFF
        assert np.all(np.diff(s.astype(int)) > 0)
    assert enc["blk_off"][-1] * 32 + 32 == enc["blocks"].size
    assert enc["nseg"] * enc["seg_quads"] >= (W.shape[1] + 3) // 4


def test_q8_bits_per_weight_near_entropy():
    # with 128-quad segments the per-segment 64-bit state costs 0.125 bit/weight;
    # the automatic choice shortens segments on small matrices to fill the GPU
    rng = np.random.default_rng(5)
    W = gauss(rng, 4, (256, 4096))
    H = codec.entropy_bits(W)
    g = codec.q8_encode(W, local=False, seg_quads=128)
    l = codec.q8_encode(W, local=True, seg_quads=128)
    assert H < g["bits_per_weight"] < H + 0.3
    assert H < l["bits_per_weight"] < H + 0.5
    auto = codec.q8_encode(W, local=False)
    assert auto["seg_quads"] % 4 == 0 and auto["bits_per_weight"] < H + 0.6


def test_q8_auto_segments():
    W = np.zeros((4096, 64), np.int8)
    e = codec.q8_encode(W[:, :64], local=False)
    assert e["nseg"] == 1
    e = codec.q8_encode(np.zeros((128, 4096), np.int8), local=False)
    assert 32 <= e["seg_quads"] <= 64 and e["seg_quads"] % 4 == 0
    e = codec.q8_encode(np.zeros((11008, 4096), np.int8), local=False)
    assert e["seg_quads"] == 64
