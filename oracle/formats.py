"""Plain-numpy readers of the reference file formats (test infrastructure only).

* safetensors as written by buffered/encoder.py:473-511 (8-byte little-endian
  header length, JSON header, raw little-endian data).
* the matvansWarpPerRow ``.bin``: file header <u32 num_matrices, u32 result_hash,
  u32 max_word_count> (create_matrices_WarpPerRow.py:440-442), the vector
  <u32 len> + int8[len] + pad to 4 (:444-453), then per matrix the layout of
  CompressedMatrix.serialize (:290-318), read back like
  CompressedMatrix.deserialize (:320-350) and matvansWarpPerRow.cu:100-145.
"""
import json
import struct

import numpy as np

_ST_DTYPES = {"I8": np.int8, "U8": np.uint8, "I16": np.int16, "U16": np.uint16, "I32": np.int32,
              "U32": np.uint32, "F32": np.float32, "F64": np.float64, "I64": np.int64,
              "U64": np.uint64, "F16": np.float16}


def read_safetensors(path):
    with open(path, "rb") as f:
        blob = f.read()
    (n,) = struct.unpack_from("<Q", blob, 0)
    header = json.loads(blob[8:8 + n])
    base = 8 + n
    out = {}
    for name, meta in header.items():
        if name == "__metadata__":
            continue
        a, b = meta["data_offsets"]
        arr = np.frombuffer(blob[base + a:base + b], dtype=_ST_DTYPES[meta["dtype"]])
        out[name] = arr.reshape(meta["shape"]).copy()
    return out


def read_wpr_bin(path):
    with open(path, "rb") as f:
        blob = f.read()
    off = 0
    num, result_hash, max_word_count = struct.unpack_from("<III", blob, off)
    off += 12
    (len_v,) = struct.unpack_from("<I", blob, off)
    off += 4
    vec = np.frombuffer(blob, dtype=np.int8, count=len_v, offset=off).copy()
    off += len_v + (3 - (len_v + 3) % 4)
    mats = []
    for _ in range(num):
        rows, cols, grid = struct.unpack_from("<IIf", blob, off)
        off += 12
        cursors = np.frombuffer(blob, dtype=np.uint32, count=rows, offset=off).copy()
        off += 4 * rows
        payload_size, min_value, G = struct.unpack_from("<IbB", blob, off)
        off += 6
        cdf = np.frombuffer(blob, dtype=np.uint8, count=G + 1, offset=off).copy()
        off += G + 1
        if (G + 1) % 2 == 1:
            off += 1
        ppf = np.frombuffer(blob, dtype=np.uint8, count=256, offset=off).copy()
        off += 256
        payload = np.frombuffer(blob[off:off + 2 * payload_size], dtype="<u2").astype(np.uint16)
        off += 2 * payload_size
        if payload_size % 2 == 1:
            off += 2
        mats.append(dict(rows=rows, cols=cols, grid_spacing=grid, cursors=cursors,
                         payload_size=payload_size, min_value=min_value, G=G, cdf=cdf, ppf=ppf,
                         payload=payload))
    assert off == len(blob), f"trailing bytes in {path}: {len(blob) - off}"
    return dict(num_matrices=num, result_hash=result_hash, max_word_count=max_word_count,
                vector=vec, matrices=mats)
