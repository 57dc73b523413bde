"""Time the reference's own Python decoders on the plain-method workload (1024x1024, sigma 4), one core.

    python oracle/time_ref_python.py [--reference PATH]   (default: $MATVANS_REFERENCE, else /root/reference)

The reference's CPU decoders decode one coder at a time: DetachedAnsQuadCoder.decode (buffered/encoder.py:
228-260) for the ans-warp-rows layout and AnsCoder.pop (matvansWarpPerRow/create_matrices_WarpPerRow.py:
250-264) for matvansWarpPerRow.  Neither walks the interleaved multi-lane layouts, so this harness recovers
each row's coders from the stored layout -- AWR: the 32 stored coder states and the row's joint word stack
(encoder.py:431-447 undone); WPR: each lane's u16 stream (create_matrices_WarpPerRow.py:390-422 undone) --
and calls the reference's decoder, unchanged, for every symbol in the order the GPU kernels consume them.
The decoded matrix must equal the encoded one; the int32 product is numpy's.  Inputs are the committed
fixtures made by the reference's encoders (tests/golden/).  Needs the reference checkout, so it runs where
the fixtures were made, not on the GPU box.
"""
import argparse
import ast
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def load_reference(ref):
    sys.path.insert(0, os.path.join(ref, "buffered"))
    import encoder  # the reference module, unchanged
    # create_matrices_WarpPerRow.py runs its pipeline at import: take its class definitions only
    src = open(os.path.join(ref, "matvansWarpPerRow", "create_matrices_WarpPerRow.py")).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, (ast.ClassDef, ast.Import, ast.ImportFrom)) and
            (not isinstance(n, ast.ClassDef) or n.name == "AnsCoder")]
    ns = {}
    exec(compile(ast.Module(body=keep, type_ignores=[]), "create_matrices_WarpPerRow.py", "exec"), ns)
    return encoder, ns["AnsCoder"]


def awr_decode_reference(enc, comp, offsets, rows, cols, ppf, cum, prob):
    """Every row through the reference's DetachedAnsQuadCoder.decode."""
    W = np.empty((rows, cols), np.int8)
    ends = list(offsets[1:]) + [comp.size // 4]
    for r in range(rows):
        words = comp[4 * int(offsets[r]):4 * int(ends[r])]
        un = words.reshape(-1, 32, 4).transpose(0, 2, 1).ravel()  # undo the block transpose
        rev_bulk = np.concatenate((un[:64], un[128:]))
        buf = enc.ArrayVector(data=rev_bulk[::-1].copy())  # encode order: pop_back yields rev_bulk[0], ...
        coders = []
        for lane in range(32):
            c = enc.DetachedAnsQuadCoder(7, 32, 64)
            c.state = (int(un[96 + lane]) << 32) | int(un[64 + lane])
            coders.append(c)
        for chunk in range(cols // 128):
            for lane in range(32):
                W[r, 128 * chunk + 4 * lane:128 * chunk + 4 * lane + 4] = coders[lane].decode(ppf, cum, prob, buf)
    return W


def wpr_decode_reference(AnsCoder, payload, cursors, rows, cols, min_value, cdf, ppf):
    """Every lane stream of every row through the reference's AnsCoder.pop."""
    W = np.empty((rows, cols), np.int8)
    ends = list(cursors[1:]) + [payload.size]
    per_lane = cols // 32
    for r in range(rows):
        L = (int(ends[r]) - int(cursors[r])) // 32  # u16 words per lane (padded to the row's longest lane)
        base = int(cursors[r])
        for lane in range(32):
            idx = [base + (k // 8) * 256 + 8 * lane + k % 8 for k in range(L)]
            stored = payload[idx]
            coder = AnsCoder(8, 16, [int(w) for w in stored[::-1]], 2)
            syms = [coder.pop(cdf, ppf) for _ in range(per_lane)]
            vals = np.asarray(syms, np.int32) + int(min_value)
            # lane j owns columns 512k + 16j .. + 15 (create_matrices_WarpPerRow.py:361-366)
            for k in range(cols // 512):
                W[r, 512 * k + 16 * lane:512 * k + 16 * lane + 16] = vals[16 * k:16 * k + 16]
    return W


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MATVANS_REFERENCE") or "/root/reference")
    a = ap.parse_args()
    enc, AnsCoder = load_reference(a.reference)
    from oracle import formats
    g = os.path.join(ROOT, "tests", "golden")
    out = {"cores": 1, "workload": "1024x1024 sigma 4 (plain method), one vector"}

    z = np.load(os.path.join(g, "awr_cases.npz"))
    W = z["c1_1024x1024_W"]
    x = np.random.default_rng(1).integers(-127, 128, size=W.shape[1]).astype(np.int8)
    p, pc, pp = enc.decoder_model_from_128bit_encoder_model(int(np.asarray(z["c1_1024x1024_min"]).reshape(-1)[0]), z["c1_1024x1024_cdf"])
    t0 = time.perf_counter()
    Wd = awr_decode_reference(enc, z["c1_1024x1024_compressed"], z["c1_1024x1024_offsets"], *W.shape, p, pc, pp)
    y = Wd.astype(np.int32) @ x.astype(np.int32)
    dt = time.perf_counter() - t0
    assert np.array_equal(Wd, W), "ans-warp-rows: the reference decoder did not reproduce the matrix"
    out["ans_warp_rows_us_per_matvec"] = 1e6 * dt
    out["ans_warp_rows_int8_equiv_gbs"] = (W.size + W.shape[1] + 4 * W.shape[0]) / dt / 1e9

    f = formats.read_wpr_bin(os.path.join(g, "wpr_c1_1024.bin"))
    raw = np.load(os.path.join(g, "wpr_c1_1024.npz"))
    m = f["matrices"][0]
    t0 = time.perf_counter()
    Wd = wpr_decode_reference(AnsCoder, m["payload"], m["cursors"], m["rows"], m["cols"], m["min_value"], m["cdf"],
                              m["ppf"])
    y = Wd.astype(np.int32) @ x.astype(np.int32)
    dt = time.perf_counter() - t0
    assert np.array_equal(Wd, raw["W"]), "matvansWarpPerRow: the reference decoder did not reproduce the matrix"
    out["matvansWarpPerRow_us_per_matvec"] = 1e6 * dt
    out["matvansWarpPerRow_int8_equiv_gbs"] = (W.size + W.shape[1] + 4 * W.shape[0]) / dt / 1e9
    assert y.shape == (W.shape[0],)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
