"""Generate the golden fixtures under tests/golden/ from the reference's own encoders.

Run once, in a container that has the reference checkout, naming its root
with --reference or the MATVANS_REFERENCE environment variable:

    python tests/golden/gen_golden.py --reference PATH/TO/MatVANS

It imports the reference's Python encoders unchanged and records their outputs:

* ``awr_chain.safetensors`` -- the reference's own end-to-end pipeline for the
  "ans-warp-rows" layout (buffered/encoder.py:527-570 with --dim 256 --count 3
  --target_entropy 4 --seed 20250829): seeded matrices, the requantised chain and
  its hashes (encoder.py:23-61), compressed with compress_ans_warp_rows
  (encoder.py:394-461) and written by compress_all_matrices (encoder.py:473-511).
  ``awr_chain_raw.npz`` holds the uncompressed matrices of the same run.
* ``awr_cases.npz`` -- compress_ans_warp_rows on non-square and edge-case
  matrices (single value, 128 distinct values, sigma 2, Laplace) plus the
  1024x1024 sigma-4 matrix of the plain-method workload.
* ``aws_chain.safetensors`` / ``aws_cases.npz`` -- the same pipeline and the
  same kinds of edge cases (rows a multiple of 32) for the "ans-warp-stripes"
  layout, compressed with compress_ans_warp_stripes (encoder.py:323-391).
  ``python tests/golden/gen_golden.py aws`` regenerates only these.
* ``wpr_chain_512.bin`` -- the reference's own matvansWarpPerRow pipeline
  (create_matrices_WarpPerRow.py, seed 20250310, -w 512 -n 3 -e 5), including
  its result_hash.
* ``wpr_c1_1024.bin`` + ``wpr_c1_1024.npz`` -- the plain-method workload: a
  1024x1024 int8 matrix clamp(round(N(0, 4^2))) encoded by encode_matrix
  (create_matrices_WarpPerRow.py:353-430) and serialised with the script's own
  file writers (:440-461), with x, per-row scales and the expected int32 y.

Two deliberate deviations, both in create_matrices_WarpPerRow.py:

* encode_matrix pads each lane of the interleaved row with ``np.empty`` (:412),
  i.e. uninitialised bytes.  The generator swaps that one call for ``np.zeros``
  so that the fixture bytes are reproducible; padding words are never consumed
  by the decoder.
* create_entropy_model computes ``value - min_value + 1`` (:181) with ``value``
  an np.int8.  The script was written for NumPy 1 (value-based promotion); under
  NumPy 2 (NEP 50) the expression is evaluated in int8 and wraps once
  ``max - min > 126``, which corrupts the CDF (the script's own assertion at :185
  then fires, e.g. for the third matrix of the seed-20250310 run).  The
  generator evaluates it with ``int(value)``, i.e. with the NumPy 1 semantics
  the script was written against.

The ans-warp-rows encoder has the same NumPy 2 hazard in
``cdf[symbols - min_symbol + 1]`` (buffered/encoder.py:202-203): with int8
``symbols`` the index wraps to -128 once ``max - min == 127`` and the top symbol
is coded with a wrong probability (seen on the 128-distinct-value case).  The
generator runs DetachedAnsQuadCoder.encode with the quad widened to int64,
i.e. with NumPy 1 promotion; for every fixture whose value range is narrower
the output is byte-identical to the unpatched call.
"""
import ast
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None  # the reference checkout's root (--reference or MATVANS_REFERENCE), set by main()


def load_awr_encoder():
    sys.path.insert(0, os.path.join(REF, "buffered"))
    import encoder  # noqa: E402  (the reference module, unchanged)

    # NumPy 1 semantics for `cdf[symbols - min_symbol (+ 1)]` (encoder.py:202-203):
    # widen the int8 quad before the reference method indexes with it.
    orig = encoder.DetachedAnsQuadCoder.encode

    def encode_np1(self, symbols, min_symbol, cdf, buf):
        return orig(self, np.asarray(symbols).astype(np.int64), min_symbol, cdf, buf)

    encoder.DetachedAnsQuadCoder.encode = encode_np1
    return encoder


def run_wpr_script(w, n, entropy, workdir):
    """Execute create_matrices_WarpPerRow.py as a module with the given argv."""
    src_path = os.path.join(REF, "matvansWarpPerRow", "create_matrices_WarpPerRow.py")
    src = open(src_path).read()
    old = "interleaved_row = np.empty(max_payload_length_rows[row]*uint16Perint4,dtype=np.uint16)"
    assert src.count(old) == 1, "reference encoder changed; update the padding patch"
    src = src.replace(old, old.replace("np.empty", "np.zeros"))
    nep50 = "padded_pmf[value - min_value + 1] = prob"
    assert src.count(nep50) == 1, "reference encoder changed; update the NEP 50 patch"
    src = src.replace(nep50, "padded_pmf[int(value) - min_value + 1] = prob")
    mod = types.ModuleType("wpr_ref")
    mod.__file__ = src_path
    sys.modules["wpr_ref"] = mod
    argv, cwd = sys.argv, os.getcwd()
    sys.argv = ["create_matrices_WarpPerRow.py", "-w", str(w), "-n", str(n), "-e", str(entropy)]
    os.chdir(workdir)
    try:
        exec(compile(src, src_path, "exec"), mod.__dict__)
    finally:
        sys.argv = argv
        os.chdir(cwd)
    return mod


def gen_awr(enc):
    # (1) the reference's own pipeline, exactly as its CLI runs it
    np.random.seed(20250829)
    mats, v0, scales, hashes = enc.create_rnd_matrices_and_vec(256, 3, 4.0)
    enc.compress_all_matrices(mats, v0, scales, hashes, enc.compress_ans_warp_rows,
                              os.path.join(HERE, "awr_chain.safetensors"))
    np.savez_compressed(os.path.join(HERE, "awr_chain_raw.npz"), matrices=mats,
                        initial_vector=v0, scales=scales, hashes=hashes)

    # (2) direct calls on edge cases and the plain-method workload
    rng = np.random.default_rng(1234)
    cases = {}

    def add(name, W):
        comp, offs, min_value, cdf = enc.compress_ans_warp_rows(W, 32)
        ppf, pcum, pprob = enc.decoder_model_from_128bit_encoder_model(min_value, cdf)
        cases[name + "_W"] = W
        cases[name + "_compressed"] = comp
        cases[name + "_offsets"] = offs
        cases[name + "_min"] = np.array([min_value], dtype=np.int32)
        cases[name + "_cdf"] = cdf
        cases[name + "_ppf"] = enc.pack_4bytes(ppf)
        cases[name + "_ppf_cum"] = enc.pack_4bytes(pcum)
        cases[name + "_ppf_prob"] = enc.pack_4bytes(pprob)

    g = lambda s, shape: np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)
    add("s4_64x512", g(4.0, (64, 512)))
    add("s2_32x256", g(2.0, (32, 256)))
    add("s1_16x1024", g(1.0, (16, 1024)))
    lap = np.clip(np.round(rng.laplace(0, 3.0, size=(24, 384))), -60, 60).astype(np.int8)
    add("lap3_24x384", lap)
    add("const_8x128", np.full((8, 128), -3, dtype=np.int8))
    two = np.where(rng.random((8, 256)) < 0.97, 5, -7).astype(np.int8)
    add("two_8x256", two)
    wide = rng.integers(-64, 64, size=(16, 512)).astype(np.int8)   # exactly 128 values
    add("wide128_16x512", wide)
    add("c1_1024x1024", g(4.0, (1024, 1024)))
    np.savez_compressed(os.path.join(HERE, "awr_cases.npz"), **cases)


def gen_aws(enc):
    # (1) the reference's pipeline with the stripes compressor (same seed and sizes as the AWR chain)
    np.random.seed(20250829)
    mats, v0, scales, hashes = enc.create_rnd_matrices_and_vec(256, 3, 4.0)
    enc.compress_all_matrices(mats, v0, scales, hashes, enc.compress_ans_warp_stripes,
                              os.path.join(HERE, "aws_chain.safetensors"))

    # (2) direct calls on edge cases (rows must be a multiple of 32, encoder.py:326)
    rng = np.random.default_rng(4321)
    cases = {}

    def add(name, W):
        comp, offs, min_value, cdf = enc.compress_ans_warp_stripes(W, 32)
        ppf, pcum, pprob = enc.decoder_model_from_128bit_encoder_model(min_value, cdf)
        cases[name + "_W"] = W
        cases[name + "_compressed"] = comp
        cases[name + "_offsets"] = offs
        cases[name + "_min"] = np.array([min_value], dtype=np.int32)
        cases[name + "_cdf"] = cdf
        cases[name + "_ppf"] = enc.pack_4bytes(ppf)
        cases[name + "_ppf_cum"] = enc.pack_4bytes(pcum)
        cases[name + "_ppf_prob"] = enc.pack_4bytes(pprob)

    g = lambda s, shape: np.clip(np.round(rng.normal(0, s, size=shape)), -127, 127).astype(np.int8)
    add("s4_64x512", g(4.0, (64, 512)))
    add("s2_32x260", g(2.0, (32, 260)))
    add("s1_96x128", g(1.0, (96, 128)))
    lap = np.clip(np.round(rng.laplace(0, 3.0, size=(32, 384))), -60, 60).astype(np.int8)
    add("lap3_32x384", lap)
    add("const_32x128", np.full((32, 128), -3, dtype=np.int8))
    two = np.where(rng.random((32, 256)) < 0.97, 5, -7).astype(np.int8)
    add("two_32x256", two)
    wide = rng.integers(-64, 64, size=(32, 512)).astype(np.int8)   # exactly 128 values
    add("wide128_32x512", wide)
    add("s4_256x1024", g(4.0, (256, 1024)))
    np.savez_compressed(os.path.join(HERE, "aws_cases.npz"), **cases)


def gen_wpr(workdir):
    # (1) the reference's own pipeline: 3 square 512x512 matrices, entropy bound 5
    mod = run_wpr_script(512, 3, 5, workdir)
    src = os.path.join(workdir, "compressed_matrices_512_5bit_count3.bin")
    os.replace(src, os.path.join(HERE, "wpr_chain_512.bin"))
    np.savez_compressed(os.path.join(HERE, "wpr_chain_512_raw.npz"),
                        matrices=mod.quantized_matrices, vector=mod.vector,
                        w_deltas=mod.w_deltas, result_hash=np.array([mod.result_hash], dtype=np.uint64))

    # (2) the plain-method workload in the WPR layout (encode_matrix needs the
    #     module global `w` equal to the square size)
    mod = run_wpr_script(1024, 1, 5, workdir)
    rng = np.random.default_rng(20251203)
    W = np.clip(np.round(rng.normal(0, 4.0, size=(1024, 1024))), -127, 127).astype(np.int8)
    x = rng.integers(-127, 128, size=1024).astype(np.int8)
    scales = rng.uniform(1e-3, 1e-2, size=1024).astype(np.float32)
    y = (W.astype(np.int64) @ x.astype(np.int64)).astype(np.int32)
    cm = mod.encode_matrix(W)
    path = os.path.join(HERE, "wpr_c1_1024.bin")
    with open(path, "wb") as f:
        mod.serialize_file_header(f, 1, 0, cm.compressed_word_count())
        mod.serialize_vector(f, x)
        cm.serialize(f)
    np.savez_compressed(os.path.join(HERE, "wpr_c1_1024.npz"), W=W, x=x, scales=scales, y=y)


def main():
    global REF
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("MATVANS_REFERENCE"),
                    help="root of the reference checkout (default: $MATVANS_REFERENCE)")
    ap.add_argument("only", nargs="*", choices=["awr", "aws", "wpr"], help="fixture families (default: all)")
    a = ap.parse_args()
    if not a.reference or not os.path.isfile(os.path.join(a.reference, "buffered", "encoder.py")):
        ap.error("the reference checkout is needed: pass --reference PATH (the directory holding buffered/ "
                 "and matvansWarpPerRow/) or set MATVANS_REFERENCE")
    REF = os.path.abspath(a.reference)
    enc = load_awr_encoder()
    only = a.only
    if not only or "awr" in only:
        gen_awr(enc)
    if not only or "aws" in only:
        gen_aws(enc)
    if not only or "wpr" in only:
        with tempfile.TemporaryDirectory() as d:
            gen_wpr(d)
    for fn in sorted(os.listdir(HERE)):
        if not fn.endswith(".py"):
            print(f"{fn:32s} {os.path.getsize(os.path.join(HERE, fn)):>9d} B")


if __name__ == "__main__":
    main()
