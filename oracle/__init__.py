"""CPU oracle for the entropy-coded matvec path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this package; the product (matvans_b200) never does.

* ``liboracle.so`` (built from oracle.c by oracle/Makefile) restates the
  reference decoders in C: the ans-warp-rows (AWR) layout of
  buffered/ans-warp-rows-kernel.cu:20-204 and the matvansWarpPerRow (WPR)
  layout of matvansWarpPerRow/matvansWarpPerRow-kernel.cu:46-175, plus an
  int64-accumulated int8 matvec and the FxHash-style vector hash of
  buffered/encoder.py:8-20.
* ``formats`` parses the reference files (safetensors written by
  buffered/encoder.py:473-511 and the .bin of create_matrices_WarpPerRow.py:
  290-319, 440-461) with plain numpy, independently of the product's C++
  readers.

Parity of this oracle is pinned by tests/test_oracle_golden.py against the
fixtures in tests/golden/, which were produced by the reference's own Python
encoders (tests/golden/gen_golden.py).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(os.path.join(HERE, "oracle.c")):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        L.orc_hash_int8.argtypes = [P, i64]
        L.orc_hash_int8.restype = ctypes.c_uint32
        L.orc_matvec_i8.argtypes = [P, i64, i64, P, ctypes.c_int, P]
        L.orc_awr_decode.argtypes = [P, i64, P, i64, i64, P, P, P, P]
        L.orc_wpr_decode.argtypes = [P, i64, P, i64, i64, ctypes.c_int8, P, ctypes.c_int, P, P]
        L.orc_awr_matvec_mt.argtypes = [P, i64, P, i64, i64, P, P, P, P, ctypes.c_int, P, ctypes.c_int]
        L.orc_wpr_matvec_mt.argtypes = [P, i64, P, i64, i64, ctypes.c_int8, P, ctypes.c_int, P, P,
                                        ctypes.c_int, P, ctypes.c_int]
        L.orc_aws_decode.argtypes = [P, i64, P, i64, i64, P, P, P, P]
        L.orc_aws_matvec.argtypes = [P, i64, P, i64, i64, P, P, P, P, ctypes.c_int, P]
        L.orc_awr_encode.argtypes = [P, i64, i64, ctypes.POINTER(P), ctypes.POINTER(i64), P, P, P, P]
        L.orc_free.argtypes = [P]
        L.orc_free.restype = None
        for f in ("orc_matvec_i8", "orc_awr_decode", "orc_wpr_decode", "orc_awr_matvec_mt", "orc_awr_encode",
                  "orc_wpr_matvec_mt", "orc_aws_decode", "orc_aws_matvec"):
            getattr(L, f).restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class OracleError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise OracleError(f"{what}: oracle status {rc}")


def hash_int8(v):
    v = _c(v, np.int8)
    return int(lib().orc_hash_int8(_p(v), v.size))


def matvec_i8(W, x):
    """y[b] = W @ x[b] with int64 accumulation; x is [cols] or [B, cols]."""
    W = _c(W, np.int8)
    x2 = _c(np.atleast_2d(x), np.int8)
    y = np.empty((x2.shape[0], W.shape[0]), dtype=np.int32)
    _check(lib().orc_matvec_i8(_p(W), W.shape[0], W.shape[1], _p(x2), x2.shape[0], _p(y)), "matvec")
    return y if np.ndim(x) == 2 else y[0]


def awr_decode(compressed, offsets, rows, cols, ppf, ppf_cum, ppf_prob):
    comp = _c(compressed, np.uint32)
    offs = _c(offsets, np.uint32)
    t = [_c(a, np.uint32) for a in (ppf, ppf_cum, ppf_prob)]
    W = np.empty((rows, cols), dtype=np.int8)
    _check(lib().orc_awr_decode(_p(comp), comp.size, _p(offs), rows, cols, *[_p(a) for a in t], _p(W)),
           "awr_decode")
    return W


def awr_encode(W):
    """The reference's compress_ans_warp_rows(W, 32) with its decoder tables (buffered/encoder.py:271-320,
    394-470), restated in C: returns (compressed u32, warp_offsets u32[rows], ppf, ppf_cum, ppf_prob u32[32])."""
    W = _c(W, np.int8)
    rows, cols = W.shape
    comp = ctypes.c_void_p()
    n = ctypes.c_int64()
    offs = np.empty(rows, np.uint32)
    t = [np.empty(32, np.uint32) for _ in range(3)]
    _check(lib().orc_awr_encode(_p(W), rows, cols, ctypes.byref(comp), ctypes.byref(n), _p(offs),
                                *[_p(a) for a in t]), "awr_encode")
    try:
        out = np.ctypeslib.as_array(ctypes.cast(comp, ctypes.POINTER(ctypes.c_uint32)), shape=(n.value,)).copy()
    finally:
        lib().orc_free(comp)
    return out, offs, t[0], t[1], t[2]


def awr_matvec(compressed, offsets, rows, cols, ppf, ppf_cum, ppf_prob, x, nthreads=1):
    comp = _c(compressed, np.uint32)
    offs = _c(offsets, np.uint32)
    t = [_c(a, np.uint32) for a in (ppf, ppf_cum, ppf_prob)]
    x2 = _c(np.atleast_2d(x), np.int8)
    y = np.empty((x2.shape[0], rows), dtype=np.int32)
    _check(lib().orc_awr_matvec_mt(_p(comp), comp.size, _p(offs), rows, cols, *[_p(a) for a in t],
                                   _p(x2), x2.shape[0], _p(y), nthreads), "awr_matvec")
    return y if np.ndim(x) == 2 else y[0]


def aws_decode(compressed, offsets, rows, cols, ppf, ppf_cum, ppf_prob):
    """'ans-warp-stripes' layout (buffered/ans-warp-stripes-kernel.cu:21-227): one offset per 32-row stripe."""
    comp = _c(compressed, np.uint32)
    offs = _c(offsets, np.uint32)
    t = [_c(a, np.uint32) for a in (ppf, ppf_cum, ppf_prob)]
    W = np.empty((rows, cols), dtype=np.int8)
    _check(lib().orc_aws_decode(_p(comp), comp.size, _p(offs), rows, cols, *[_p(a) for a in t], _p(W)),
           "aws_decode")
    return W


def aws_matvec(compressed, offsets, rows, cols, ppf, ppf_cum, ppf_prob, x):
    comp = _c(compressed, np.uint32)
    offs = _c(offsets, np.uint32)
    t = [_c(a, np.uint32) for a in (ppf, ppf_cum, ppf_prob)]
    x2 = _c(np.atleast_2d(x), np.int8)
    y = np.empty((x2.shape[0], rows), dtype=np.int32)
    _check(lib().orc_aws_matvec(_p(comp), comp.size, _p(offs), rows, cols, *[_p(a) for a in t],
                                _p(x2), x2.shape[0], _p(y)), "aws_matvec")
    return y if np.ndim(x) == 2 else y[0]


def wpr_decode(payload, cursors, rows, cols, min_value, cdf, ppf):
    pay = _c(payload, np.uint16)
    cur = _c(cursors, np.uint32)
    cdf = _c(cdf, np.uint8)
    ppf = _c(ppf, np.uint8)
    W = np.empty((rows, cols), dtype=np.int8)
    _check(lib().orc_wpr_decode(_p(pay), pay.size, _p(cur), rows, cols, int(min_value), _p(cdf),
                                cdf.size - 1, _p(ppf), _p(W)), "wpr_decode")
    return W


def wpr_matvec(payload, cursors, rows, cols, min_value, cdf, ppf, x, nthreads=1):
    pay = _c(payload, np.uint16)
    cur = _c(cursors, np.uint32)
    cdf = _c(cdf, np.uint8)
    ppf = _c(ppf, np.uint8)
    x2 = _c(np.atleast_2d(x), np.int8)
    y = np.empty((x2.shape[0], rows), dtype=np.int32)
    _check(lib().orc_wpr_matvec_mt(_p(pay), pay.size, _p(cur), rows, cols, int(min_value), _p(cdf),
                                   cdf.size - 1, _p(ppf), _p(x2), x2.shape[0], _p(y), nthreads),
           "wpr_matvec")
    return y if np.ndim(x) == 2 else y[0]
