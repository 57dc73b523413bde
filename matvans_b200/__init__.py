"""matvans_b200: entropy-coded int8 matrix-vector products on NVIDIA B200 (sm_100a).

Int8 weight matrices are stored as interleaved rANS streams and decoded inside
the matvec kernel.  Layouts: the reference's ans-warp-rows (safetensors) and
matvansWarpPerRow (.bin) formats, and this library's Q8-stripe layout with
global or per-row tables.

    from matvans_b200 import codec, ops
    M = ops.Q8Matrix.encode(W)          # W: int8 numpy [rows, cols]
    y = M.matvec(x)                      # x: int8 [cols] or [B, cols]; y: exact int32

The C ABI is include/matvans.h; libmatvans.so is built in-tree by
``python -m matvans_b200.build``.
"""
from ._lib import LIB_PATH, MatvansError, lib  # noqa: F401

__version__ = "0.1.0"


def version():
    return lib().mv_version().decode()
