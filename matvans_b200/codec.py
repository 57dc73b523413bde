"""Host-side codec API: the reference's encoder functions, same names and
results, backed by the C++ encoders of libmatvans.so.

Mirrors (paths within the reference project):
  buffered/encoder.py:8-20      hash_int8_array
  buffered/encoder.py:271-306   fit_128bit_encoder_model
  buffered/encoder.py:309-320   decoder_model_from_128bit_encoder_model
  buffered/encoder.py:394-461   compress_ans_warp_rows
  buffered/encoder.py:464-470   pack_4bytes
  buffered/encoder.py:473-511   compress_all_matrices
  matvansWarpPerRow/create_matrices_WarpPerRow.py:131-187  create_entropy_model
  matvansWarpPerRow/create_matrices_WarpPerRow.py:189-208  create_ppf
  matvansWarpPerRow/create_matrices_WarpPerRow.py:274-350  CompressedMatrix
  matvansWarpPerRow/create_matrices_WarpPerRow.py:353-430  encode_matrix
plus the Q8-stripe encoder of this library (q8_encode).
"""
import ctypes
import struct
import sys

import numpy as np

from . import _lib
from ._lib import Blob, check, lib, ptr


def _i8(a, name="matrix"):
    a = np.asarray(a)
    if a.dtype != np.int8:
        raise TypeError(f"{name} must be int8, got {a.dtype}")
    return np.ascontiguousarray(a)


def hash_int8_array(arr):
    """FxHash-style hash of an int8 array (buffered/encoder.py:8-20)."""
    a = _i8(arr, "arr").ravel()
    return int(lib().mv_hash_int8(ptr(a), a.size))


def entropy_bits(data):
    """Empirical entropy in bits per element of an int8 array."""
    _, counts = np.unique(np.asarray(data), return_counts=True)
    p = counts / counts.sum()
    return float(-(p * np.log2(p)).sum())


# ------------------------------------------------------------------ AWR

def _awr_blob(matrix, nthreads=0):
    W = _i8(matrix)
    if W.ndim != 2:
        raise ValueError("matrix must have rank 2")
    h = _lib.new_blob_out()
    check(lib().mv_awr_encode(ptr(W), W.shape[0], W.shape[1], nthreads, ctypes.byref(h)))
    return Blob(h.value)


def compress_ans_warp_rows(matrix, warp_size=32):
    """Returns (compressed u32, warp_offsets u32 [rows] in uint4 units, min_value, cdf u8),
    byte-identical to buffered/encoder.py:394-461."""
    if warp_size != 32:
        raise ValueError("the ans-warp-rows layout is defined for warp_size 32")
    b = _awr_blob(matrix)
    return (b.array("compressed", np.uint32), b.array("warp_offsets", np.uint32), b.scalar("min_value"),
            b.array("cdf", np.uint8))


def compress_ans_warp_stripes(matrix, warp_size=32):
    """Returns (compressed u32, warp_offsets u32 [rows/32] in uint4 units, min_value, cdf u8),
    byte-identical to buffered/encoder.py:323-391 (rows % 32 == 0, cols % 4 == 0)."""
    if warp_size != 32:
        raise ValueError("the ans-warp-stripes layout is defined for warp_size 32")
    W = _i8(matrix)
    if W.ndim != 2:
        raise ValueError("matrix must have rank 2")
    h = _lib.new_blob_out()
    check(lib().mv_aws_encode(ptr(W), W.shape[0], W.shape[1], 0, ctypes.byref(h)))
    b = Blob(h.value)
    return (b.array("compressed", np.uint32), b.array("warp_offsets", np.uint32), b.scalar("min_value"),
            b.array("cdf", np.uint8))


def fit_128bit_encoder_model(data):
    """(entropy, cross_entropy, min_value, cdf) as buffered/encoder.py:271-306.

    The same model is fitted in C++ by mv_awr_encode; this mirror exists for
    callers that want the model (and its entropy figures) without encoding."""
    data = _i8(data, "data")
    values, counts = np.unique(data, return_counts=True)
    numel = data.size
    c32 = counts.astype(np.float32)
    pmf = np.maximum(1, np.round(c32 * 128 / numel).astype(np.uint32))
    s = int(pmf.sum())
    for _ in range(max(0, s - 128)):
        pmf[np.argmax(pmf)] -= 1
    for _ in range(max(0, 128 - s)):
        pmf[np.argmax(pmf)] += 1
    entropy = np.log2(numel) - np.sum(c32 * np.log2(c32)) / numel
    cross_entropy = 7 - np.sum(c32 * np.log2(pmf)) / numel
    min_value, max_value = int(values[0]), int(values[-1])
    cdf = np.zeros(max_value - min_value + 2, dtype=np.uint8)
    left, last = 0, 0
    for v, f in zip(values, pmf):
        idx = int(v) - min_value
        cdf[last + 1:idx + 1] = left
        last = idx
        left += int(f)
    if left != 128:
        raise ValueError("model does not sum to 128")
    cdf[-1] = 128
    return entropy, cross_entropy, min_value, cdf


def decoder_model_from_128bit_encoder_model(min_value, cdf):
    """(ppf int8[128], ppf_cum u8[128], ppf_prob u8[128]), buffered/encoder.py:309-320."""
    ppf = np.zeros(128, np.int8)
    ppf_cum = np.zeros(128, np.uint8)
    ppf_prob = np.zeros(128, np.uint8)
    cdf = np.asarray(cdf)
    for index, (lc, rc) in enumerate(zip(cdf[:-1], cdf[1:])):
        ppf[int(lc):int(rc)] = index + min_value
        ppf_cum[int(lc):int(rc)] = lc
        ppf_prob[int(lc):int(rc)] = int(rc) - int(lc)
    return ppf, ppf_cum, ppf_prob


def pack_4bytes(arr):
    """Little-endian packing of 4n bytes into n u32 (buffered/encoder.py:464-470)."""
    a = np.asarray(arr)
    assert a.dtype in (np.uint8, np.int8) and a.ndim == 1
    return a.astype(np.uint8).reshape(-1, 4).view("<u4").ravel().astype(np.uint32)


def compress_all_matrices(matrices, initial_vector, scales, hashes, compressor, filename):
    """Writes the safetensors file of buffered/encoder.py:473-511 (compressor:
    compress_ans_warp_rows or compress_ans_warp_stripes)."""
    if compressor not in (compress_ans_warp_rows, compress_ans_warp_stripes):
        raise ValueError("compressor must be compress_ans_warp_rows or compress_ans_warp_stripes")
    comp, offs, ppfs, cums, probs = [], [], [], [], []
    size = 0
    for m in matrices:
        c, o, mn, cdf = compressor(m, 32)
        p, pc, pp = decoder_model_from_128bit_encoder_model(mn, cdf)
        comp.append(c)
        offs.append(o + size)
        ppfs.append(pack_4bytes(p))
        cums.append(pack_4bytes(pc))
        probs.append(pack_4bytes(pp))
        size += len(c) // 4
    tensors = {
        "initial_vector": _i8(initial_vector, "initial_vector"),
        "scales": np.asarray(scales, np.float32),
        "hashes": np.asarray(hashes, np.uint32),
        "compressed": np.concatenate(comp),
        "all_warp_offsets": np.stack(offs),
        "all_ppfs": np.stack(ppfs),
        "all_ppfs_cum": np.stack(cums),
        "all_ppfs_prob": np.stack(probs),
    }
    save_safetensors(filename, tensors)


# ------------------------------------------------------------------ WPR

def create_entropy_model(data, precision=8):
    """(min_value, grid_size, cdf u16, entropy, cross_entropy): the model of
    create_matrices_WarpPerRow.py:131-187 (stable tie order, see host_ref_encoders.cpp)."""
    if precision != 8:
        raise ValueError("the WPR layout uses 8-bit precision")
    data = _i8(data, "data")
    mn, mx = int(data.min()), int(data.max())
    if mn == mx:
        return mn, 2, np.array([0, 255, 256], np.uint16), 0.0, float(-np.log1p(-1 / 256) / np.log(2))
    values, counts = np.unique(data, return_counts=True)
    order = np.argsort(counts, kind="stable")[::-1]
    values, counts = values[order], counts[order]
    q = np.maximum(1, np.round(counts * (256 / data.size)).astype(np.uint16))
    excess = int(q.sum()) - 256
    if excess > 0:
        while excess > 0:
            n = min(excess, int((q > 1).sum()))
            q[:n] -= 1
            excess -= n
    elif excess < 0:
        q[excess:] += 1
    grid = mx - mn + 1
    pmf = np.zeros(grid + 1, np.uint16)
    for v, p in zip(values, q):
        pmf[int(v) - mn + 1] = p
    cdf = np.cumsum(pmf, dtype=np.uint16)
    entropy = np.log2(data.size) - (counts @ np.log2(counts)) / data.size
    cross_entropy = 8 - (counts @ np.log2(q.astype(np.float64))) / data.size
    return mn, grid, cdf, float(entropy), float(cross_entropy)


def create_ppf(cdf, p_precision=8):
    """ppf u8[256] of create_matrices_WarpPerRow.py:189-208."""
    cdf = np.asarray(cdf)
    ppf = np.zeros(1 << p_precision, np.uint8)
    low = (cdf & 0xFF).astype(np.uint8)
    for p in range(1 << p_precision):
        for r in range(len(cdf) - 1, 0, -1):
            if low[r - 1] <= p:
                ppf[p] = r - 1
                break
    return ppf


def _wpr_blob(matrix, nthreads=0):
    W = _i8(matrix)
    h = _lib.new_blob_out()
    check(lib().mv_wpr_encode(ptr(W), W.shape[0], W.shape[1], nthreads, ctypes.byref(h)))
    return Blob(h.value)


class CompressedMatrix:
    """One WPR matrix (create_matrices_WarpPerRow.py:274-350)."""

    def __init__(self, rows, cols, grid_spacing, cursors, min_value, cdf, ppf, payload):
        self.rows, self.cols, self.grid_spacing = int(rows), int(cols), float(grid_spacing)
        self.cursors = np.asarray(cursors, np.uint32)
        self.min_value = int(min_value)
        self.cdf = (np.asarray(cdf) & 0xFF).astype(np.uint8)
        self.ppf = (np.asarray(ppf) & 0xFF).astype(np.uint8)
        self.payload = np.asarray(payload, np.uint16)

    @property
    def G(self):
        return len(self.cdf) - 1

    def compressed_word_count(self):
        even = len(self.payload) + len(self.payload) % 2
        return (4 + self.rows) * 2 + (3 + len(self.cdf)) // 2 + even

    def serialize(self, f):
        f.write(struct.pack(f"<LLf{self.rows}LLbB{len(self.cdf)}B", self.rows, self.cols, self.grid_spacing,
                            *self.cursors.tolist(), len(self.payload), self.min_value, len(self.cdf) - 1,
                            *self.cdf.tolist()))
        if len(self.cdf) % 2 == 1:
            f.write(b"\0")
        f.write(struct.pack("<256B", *self.ppf.tolist()))
        f.write(self.payload.astype("<u2").tobytes())
        if len(self.payload) % 2 == 1:
            f.write(b"\0\0")


def encode_matrix(matrix, precision=8):
    """WPR encoding of an int8 matrix (create_matrices_WarpPerRow.py:353-430)."""
    if precision != 8:
        raise ValueError("the WPR layout uses 8-bit precision")
    b = _wpr_blob(matrix)
    return CompressedMatrix(b.scalar("rows"), b.scalar("cols"), 1.0, b.array("cursors", np.uint32),
                            b.scalar("min_value"), b.array("cdf", np.uint8), b.array("ppf", np.uint8),
                            b.array("payload", np.uint16))


def write_wpr_bin(path, matrices, vector, result_hash=0):
    """The .bin file of create_matrices_WarpPerRow.py:440-461."""
    vector = _i8(vector, "vector")
    with open(path, "wb") as f:
        mwc = max(m.compressed_word_count() for m in matrices)
        f.write(struct.pack("<LLL", len(matrices), result_hash, mwc))
        f.write(struct.pack("<L", len(vector)))
        f.write(vector.tobytes())
        f.write(b"\0" * (3 - (len(vector) + 3) % 4))
        for m in matrices:
            m.serialize(f)


def read_wpr_bin(path):
    """Reads a .bin file with the C++ reader; returns (header dict, vector, [CompressedMatrix])."""
    h = _lib.new_blob_out()
    check(lib().mv_read_wpr_bin(str(path).encode(), ctypes.byref(h)))
    b = Blob(h.value)
    hdr = {k: b.scalar(k) for k in ("num_matrices", "result_hash", "max_word_count", "len_v")}
    mats = []
    for i in range(hdr["num_matrices"]):
        p = f"m{i}."
        mats.append(CompressedMatrix(b.scalar(p + "rows"), b.scalar(p + "cols"), 1.0,
                                     b.array(p + "cursors", np.uint32), b.scalar(p + "min_value"),
                                     b.array(p + "cdf", np.uint8), b.array(p + "ppf", np.uint8),
                                     b.array(p + "payload", np.uint16)))
    return hdr, b.array("vector", np.int8), mats


# ------------------------------------------------------------- safetensors

def load_safetensors(path):
    """All tensors of a safetensors file, read by the C++ parser (replaces
    SaneSafetensorFile, buffered/sane_safetensors.hpp:17-68)."""
    h = _lib.new_blob_out()
    check(lib().mv_read_safetensors(str(path).encode(), ctypes.byref(h)))
    b = Blob(h.value)
    return {n: b.array(n) for n in b.names()}


def save_safetensors(path, tensors):
    """Write numpy arrays as a safetensors file (the byte layout mv_write_safetensors writes)."""
    import json
    names = list(tensors)
    header, off, chunks = {}, 0, []
    codes = {np.int8: "I8", np.uint8: "U8", np.int16: "I16", np.uint16: "U16", np.int32: "I32",
             np.uint32: "U32", np.float32: "F32", np.int64: "I64", np.uint64: "U64", np.float64: "F64"}
    for n in names:
        a = np.ascontiguousarray(tensors[n])
        code = codes[a.dtype.type]
        raw = a.astype(a.dtype.newbyteorder("<")).tobytes()
        header[n] = {"dtype": code, "shape": list(a.shape), "data_offsets": [off, off + len(raw)]}
        off += len(raw)
        chunks.append(raw)
    h = json.dumps(header, separators=(",", ":")).encode()
    h += b" " * ((8 - (8 + len(h)) % 8) % 8)
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(h)))
        f.write(h)
        for c in chunks:
            f.write(c)


# -------------------------------------------------------------------- Q8

def q8_encode(matrix, local=True, seg_quads=0, nthreads=0):
    """Encode an int8 matrix in the Q8-stripe layout.  Returns a dict of host
    arrays and metadata (see mv_q8_view in include/matvans.h)."""
    W = _i8(matrix)
    if W.ndim != 2:
        raise ValueError("matrix must have rank 2")
    h = _lib.new_blob_out()
    check(lib().mv_q8_encode(ptr(W), W.shape[0], W.shape[1], int(bool(local)), int(seg_quads), int(nthreads),
                             ctypes.byref(h)))
    b = Blob(h.value)
    out = {k: b.array(k) for k in ("blocks", "blk_off", "tbl", "tbl_off")}
    for k in ("rows", "cols", "seg_quads", "nseg", "local", "max_blk_rows", "tbl_stripe_max", "payload_bytes",
              "stream_bytes"):
        out[k] = b.scalar(k)
    out["bits_per_weight"] = 8.0 * out["payload_bytes"] / (out["rows"] * out["cols"])
    return out


_Q8_KEYS = ("rows", "cols", "seg_quads", "nseg", "local", "max_blk_rows", "tbl_stripe_max")


def save_q8(path, encodings, row_scales=None, chain=None):
    """Write Q8 encodings (dicts from q8_encode) as one safetensors file (mv_q8_save).  row_scales: optional
    list of per-row fp32 arrays (None entries allowed); chain: optional dict with "initial_vector" (int8),
    "scales" (fp32 per matrix) and "hashes" (u32 per matrix), stored under the reference's tensor names."""
    keep, hosts = [], (_lib.Q8Host * len(encodings))()
    for i, e in enumerate(encodings):
        arrs = [np.ascontiguousarray(e["blocks"], np.uint32), np.ascontiguousarray(e["blk_off"], np.uint32),
                np.ascontiguousarray(e["tbl"], np.uint16), np.ascontiguousarray(e["tbl_off"], np.uint32)]
        sc = None if row_scales is None or row_scales[i] is None else np.ascontiguousarray(row_scales[i], np.float32)
        if sc is not None and sc.shape != (int(e["rows"]),):
            raise ValueError(f"row_scales[{i}] must have {e['rows']} entries")
        keep += arrs + ([sc] if sc is not None else [])
        h = hosts[i]
        h.blocks, h.blk_off, h.tbl, h.tbl_off = [a.ctypes.data for a in arrs]
        h.n_blocks, h.n_blk_off, h.n_tbl, h.n_tbl_off = [a.size for a in arrs]
        for k in _Q8_KEYS:
            setattr(h, k, int(e[k]))
        h.row_scales = sc.ctypes.data if sc is not None else None
    ch = None
    if chain:
        ch = _lib.Q8ChainHost()
        for k, dt in (("initial_vector", np.int8), ("scales", np.float32), ("hashes", np.uint32)):
            if chain.get(k) is not None:
                a = np.ascontiguousarray(chain[k], dt)
                if k != "initial_vector" and a.size != len(encodings):
                    raise ValueError(f"chain {k} needs one entry per matrix")
                keep.append(a)
                setattr(ch, k, a.ctypes.data)
                if k == "initial_vector":
                    ch.n_initial = a.size
    check(lib().mv_q8_save(str(path).encode(), hosts, len(encodings), ctypes.byref(ch) if ch else None))


def load_q8(path):
    """Read a Q8 file written by save_q8 / mv_q8_save: (encodings, row_scales, chain).  encodings are dicts in
    q8_encode's form (host arrays), row_scales a list of fp32 arrays or None, chain a dict (entries None when
    absent).  The file is checked against the layout's shape rules (mv_q8_file_matrix)."""
    h = _lib.new_blob_out()
    check(lib().mv_read_safetensors(str(path).encode(), ctypes.byref(h)))
    b = Blob(h.value)
    n = ctypes.c_int32()
    check(lib().mv_q8_file_count(b._h, ctypes.byref(n)))
    encs, scales = [], []

    def grab(p, cnt, dt):
        if not p or not cnt:
            return np.zeros(0, dt)
        buf = (ctypes.c_char * (cnt * np.dtype(dt).itemsize)).from_address(p)
        return np.frombuffer(buf, dtype=dt).copy()
    for i in range(n.value):
        q = _lib.Q8Host()
        check(lib().mv_q8_file_matrix(b._h, i, ctypes.byref(q)))
        e = {k: int(getattr(q, k)) for k in _Q8_KEYS}
        e["blocks"] = grab(q.blocks, q.n_blocks, np.uint32)
        e["blk_off"] = grab(q.blk_off, q.n_blk_off, np.uint32)
        e["tbl"] = grab(q.tbl, q.n_tbl, np.uint16)
        e["tbl_off"] = grab(q.tbl_off, q.n_tbl_off, np.uint32)
        e["payload_bytes"] = (4 * int(e["blk_off"][-1]) * 32 + 2 * e["tbl"].size + 4 * e["tbl_off"].size +
                              4 * e["blk_off"].size)
        e["bits_per_weight"] = 8.0 * e["payload_bytes"] / (e["rows"] * e["cols"])
        encs.append(e)
        scales.append(grab(q.row_scales, e["rows"], np.float32) if q.row_scales else None)
    c = _lib.Q8ChainHost()
    check(lib().mv_q8_file_chain(b._h, ctypes.byref(c)))
    chain = {"initial_vector": grab(c.initial_vector, c.n_initial, np.int8) if c.initial_vector else None,
             "scales": grab(c.scales, n.value, np.float32) if c.scales else None,
             "hashes": grab(c.hashes, n.value, np.uint32) if c.hashes else None}
    return encs, scales, chain


__all__ = [n for n in dir() if not n.startswith("_")]
if sys.byteorder != "little":  # pragma: no cover
    raise ImportError("matvans_b200 assumes a little-endian host, like the reference")
