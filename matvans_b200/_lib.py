"""ctypes binding of libmatvans.so (the C ABI declared in include/matvans.h).

The shared library is built in-tree by ``python -m matvans_b200.build`` (or
``__graft_entry__.build()``).  Nothing here falls back to another
implementation: if the library is missing, loading raises.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmatvans.so")

MV_OK = 0
STATUS_NAMES = {1: "MV_ERR_ARG", 2: "MV_ERR_SHAPE", 3: "MV_ERR_FORMAT", 4: "MV_ERR_IO", 5: "MV_ERR_CUDA",
                6: "MV_ERR_DEVICE", 7: "MV_ERR_NOMEM", 8: "MV_ERR_UNSUPPORTED"}
DEV_STREAM_OVERRUN, DEV_FINAL_STATE, DEV_WAIT_TIMEOUT, DEV_BAD_TABLE = 1, 2, 4, 8
# integer batches of at least this many vectors run on the tensor cores with engine 0
# (MV_MMA_MIN_VECTORS in include/matvans.h); smaller ones always use dp4a
MMA_MIN_BATCH = 3

# every symbol include/matvans.h declares
EXPORTS = [
    "mv_version", "mv_last_error", "mv_device_status", "mat_vec_mul_coalesced", "mv_awr_matvec",
    "mv_awr_matvec_requant", "mv_wpr_matvec", "mv_requant_absmax", "mv_q8_matvec", "mv_q8_decode",
    "mv_dense_matvec", "mv_blob_free", "mv_blob_get", "mv_blob_get_i64", "mv_blob_name", "mv_awr_encode",
    "mv_wpr_encode", "mv_q8_encode", "mv_read_safetensors", "mv_write_safetensors", "mv_read_wpr_bin",
    "mv_hash_int8", "mv_debug_inject", "mv_requant_absmax_noalloc", "mv_q8_matvec_tuned", "mv_q8_stack_plan",
    "mv_q8_stack_matvec", "mv_q8_matvec_bf16", "mv_q8_matvec_t_bf16", "mv_q8_chain_plan", "mv_q8_chain_matvec",
    "mv_aws_matvec", "mv_aws_matvec_requant", "mv_aws_encode", "mat_vec_mul_coalesced_stripes",
    "mv_q8_x_tiles_bytes", "mv_debug_query", "mv_q8_save", "mv_q8_file_count", "mv_q8_file_matrix",
    "mv_q8_file_chain", "mv_q8_upload", "mv_q8_load", "mv_q8_matrix_view", "mv_q8_matrix_row_scales",
    "mv_q8_matrix_free",
]


class MatvansError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Q8View(ctypes.Structure):
    """struct mv_q8_view (include/matvans.h)."""
    _fields_ = [("blocks", ctypes.c_void_p), ("blk_off", ctypes.c_void_p), ("tbl", ctypes.c_void_p),
                ("tbl_off", ctypes.c_void_p), ("rows", ctypes.c_int32), ("cols", ctypes.c_int32),
                ("seg_quads", ctypes.c_int32), ("nseg", ctypes.c_int32), ("local", ctypes.c_int32),
                ("max_blk_rows", ctypes.c_int32), ("blocks_rows", ctypes.c_uint32),
                ("tbl_len", ctypes.c_uint32), ("tbl_stripe_max", ctypes.c_uint32)]


class Q8Host(ctypes.Structure):
    """struct mv_q8_host."""
    _fields_ = [("blocks", ctypes.c_void_p), ("n_blocks", ctypes.c_size_t), ("blk_off", ctypes.c_void_p),
                ("n_blk_off", ctypes.c_size_t), ("tbl", ctypes.c_void_p), ("n_tbl", ctypes.c_size_t),
                ("tbl_off", ctypes.c_void_p), ("n_tbl_off", ctypes.c_size_t), ("rows", ctypes.c_int32),
                ("cols", ctypes.c_int32), ("seg_quads", ctypes.c_int32), ("nseg", ctypes.c_int32),
                ("local", ctypes.c_int32), ("max_blk_rows", ctypes.c_int32), ("tbl_stripe_max", ctypes.c_uint32),
                ("row_scales", ctypes.c_void_p)]


class Q8ChainHost(ctypes.Structure):
    """struct mv_q8_chain_host."""
    _fields_ = [("initial_vector", ctypes.c_void_p), ("n_initial", ctypes.c_size_t), ("scales", ctypes.c_void_p),
                ("hashes", ctypes.c_void_p)]


class Q8Tuning(ctypes.Structure):
    """struct mv_q8_tuning."""
    _fields_ = [("warps", ctypes.c_int32), ("ilp", ctypes.c_int32), ("depth", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("parts", ctypes.c_int32), ("engine", ctypes.c_int32)]


class Q8Job(ctypes.Structure):
    """struct mv_q8_job."""
    _fields_ = [("m", Q8View), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("scales", ctypes.c_void_p),
                ("ys", ctypes.c_void_p), ("ngroups", ctypes.c_int32), ("atomic", ctypes.c_int32),
                ("item0", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("x_tiles", ctypes.c_void_p)]


class Q8StackInfo(ctypes.Structure):
    """struct mv_q8_stack_info."""
    _fields_ = [("nitems", ctypes.c_uint32), ("max_blk_rows", ctypes.c_int32), ("tbl_stripe_max", ctypes.c_uint32),
                ("warps", ctypes.c_int32), ("ilp", ctypes.c_int32), ("depth", ctypes.c_int32),
                ("atomic_jobs", ctypes.c_int32)]


_LIB = None


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m matvans_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, i32, sz, u32p = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p
    st = ctypes.c_int
    sig = {
        "mv_version": ([], ctypes.c_char_p),
        "mv_last_error": ([], ctypes.c_char_p),
        "mv_device_status": ([P, ctypes.POINTER(ctypes.c_uint32)], st),
        "mat_vec_mul_coalesced": ([P, P, sz, sz, ctypes.c_float, P, P, P, P, P], None),
        "mv_awr_matvec": ([P, sz, P, P, P, P, i32, i32, P, i32, P, P, P, P], st),
        "mv_awr_matvec_requant": ([P, sz, P, P, P, P, i32, i32, P, ctypes.c_float, P, P], st),
        "mat_vec_mul_coalesced_stripes": ([P, P, sz, sz, ctypes.c_float, P, P, P, P, P], None),
        "mv_aws_matvec": ([P, sz, P, P, P, P, i32, i32, P, i32, P, P, P, P], st),
        "mv_aws_matvec_requant": ([P, sz, P, P, P, P, i32, i32, P, ctypes.c_float, P, P], st),
        "mv_wpr_matvec": ([P, sz, P, ctypes.c_int8, P, i32, P, i32, i32, P, i32, P, P, P, P], st),
        "mv_requant_absmax": ([P, i32, P, P, P, P], st),
        "mv_requant_absmax_noalloc": ([P, i32, P, P, P], st),
        "mv_q8_matvec": ([ctypes.POINTER(Q8View), P, i32, P, P, P, P], st),
        "mv_q8_decode": ([ctypes.POINTER(Q8View), P, P], st),
        "mv_q8_matvec_tuned": ([ctypes.POINTER(Q8View), P, i32, P, P, P, ctypes.POINTER(Q8Tuning), P], st),
        "mv_q8_stack_plan": ([ctypes.POINTER(Q8Job), i32, ctypes.POINTER(Q8Tuning), ctypes.POINTER(Q8StackInfo)], st),
        "mv_q8_stack_matvec": ([P, i32, ctypes.POINTER(Q8StackInfo), i32, ctypes.POINTER(Q8Tuning), P], st),
        "mv_q8_x_tiles_bytes": ([ctypes.POINTER(Q8View)], sz),
        "mv_q8_chain_plan": ([ctypes.POINTER(Q8Job), i32, ctypes.POINTER(Q8Tuning), ctypes.POINTER(Q8StackInfo)], st),
        "mv_q8_chain_matvec": ([P, i32, ctypes.POINTER(Q8StackInfo), i32, P, P, ctypes.POINTER(Q8Tuning), P], st),
        "mv_q8_matvec_bf16": ([ctypes.POINTER(Q8View), P, i32, P, P, ctypes.POINTER(Q8Tuning), P], st),
        "mv_q8_matvec_t_bf16": ([ctypes.POINTER(Q8View), P, i32, P, P, ctypes.POINTER(Q8Tuning), P], st),
        "mv_dense_matvec": ([P, i32, i32, P, i32, P, P], st),
        "mv_blob_free": ([P], None),
        "mv_blob_get": ([P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)], st),
        "mv_blob_get_i64": ([P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)], st),
        "mv_blob_name": ([P, i32], ctypes.c_char_p),
        "mv_awr_encode": ([P, i32, i32, i32, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_aws_encode": ([P, i32, i32, i32, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_wpr_encode": ([P, i32, i32, i32, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_q8_encode": ([P, i32, i32, i32, i32, i32, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_read_safetensors": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_write_safetensors": ([ctypes.c_char_p, P], st),
        "mv_read_wpr_bin": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_hash_int8": ([P, sz], ctypes.c_uint32),
        "mv_debug_inject": ([i32, ctypes.c_uint32], st),
        "mv_debug_query": ([i32, ctypes.POINTER(ctypes.c_uint64)], st),
        "mv_q8_save": ([ctypes.c_char_p, ctypes.POINTER(Q8Host), i32, ctypes.POINTER(Q8ChainHost)], st),
        "mv_q8_file_count": ([P, ctypes.POINTER(i32)], st),
        "mv_q8_file_matrix": ([P, i32, ctypes.POINTER(Q8Host)], st),
        "mv_q8_file_chain": ([P, ctypes.POINTER(Q8ChainHost)], st),
        "mv_q8_upload": ([ctypes.POINTER(Q8Host), ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_q8_load": ([ctypes.c_char_p, i32, ctypes.POINTER(ctypes.c_void_p)], st),
        "mv_q8_matrix_view": ([P], ctypes.POINTER(Q8View)),
        "mv_q8_matrix_row_scales": ([P], P),
        "mv_q8_matrix_free": ([P], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def check(rc):
    if rc != MV_OK:
        raise MatvansError(rc, lib().mv_last_error().decode())


# ---------------------------------------------------------------- blobs

_DT = {1: np.int8, 2: np.uint8, 3: np.int16, 4: np.uint16, 5: np.int32, 6: np.uint32, 7: np.float32,
       8: np.int64, 9: np.uint64, 10: np.float64}
_DT_CODE = {np.dtype(v): k for k, v in _DT.items()}


class Blob:
    """Host arrays + scalars produced by an encoder or a file reader."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _LIB is not None:
            _LIB.mv_blob_free(self._h)
            self._h = ctypes.c_void_p(0)

    def names(self):
        out, i = [], 0
        while True:
            n = lib().mv_blob_name(self._h, i)
            if n is None:
                return out
            out.append(n.decode())
            i += 1

    def scalar(self, name):
        v = ctypes.c_int64()
        check(lib().mv_blob_get_i64(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    def has_scalar(self, name):
        v = ctypes.c_int64()
        return lib().mv_blob_get_i64(self._h, name.encode(), ctypes.byref(v)) == MV_OK

    def array(self, name, dtype=None):
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        check(lib().mv_blob_get(self._h, name.encode(), ctypes.byref(p), ctypes.byref(n)))
        if dtype is None:
            dtype = _DT[self.scalar(name + ".dtype")] if self.has_scalar(name + ".dtype") else np.uint8
        if n.value == 0:
            a = np.zeros(0, dtype=dtype)
        else:
            buf = (ctypes.c_uint8 * n.value).from_address(p.value)
            a = np.frombuffer(buf, dtype=np.uint8).copy().view(dtype)
        if self.has_scalar(name + ".ndim"):
            nd = self.scalar(name + ".ndim")
            shape = tuple(self.scalar(f"{name}.shape{i}") for i in range(nd))
            if int(np.prod(shape)) == a.size:
                a = a.reshape(shape)
        return a


def ptr(a):
    """Address of a numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def new_blob_out():
    return ctypes.c_void_p()
