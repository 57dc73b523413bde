"""Device-side API: compressed matrices resident in GPU memory and the fused
decode + matvec launches of libmatvans.so.

torch provides device memory and the current CUDA stream; every launch goes
through the C ABI.  There is no CPU or torch fallback: without a GPU or
without the built library these calls raise.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import MMA_MIN_BATCH, Q8Job, Q8StackInfo, Q8Tuning, Q8View, check, lib

_STATUS_BITS = {1: "stream overrun", 2: "final coder state mismatch", 4: "wait timeout", 8: "bad table"}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(a, device, dtype=None):
    """numpy -> device tensor (16-byte aligned by the caching allocator)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.view(dtype)
    return t.to(device)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _as_x(x, cols, device):
    if not isinstance(x, torch.Tensor):
        x = torch.from_numpy(np.ascontiguousarray(x, dtype=np.int8))
    if x.dtype != torch.int8:
        raise TypeError("x must be int8")
    squeeze = x.dim() == 1
    x2 = x.reshape(1, -1) if squeeze else x
    if x2.shape[-1] != cols:
        raise ValueError(f"x has {x2.shape[-1]} columns, matrix has {cols}")
    return x2.to(device).contiguous(), squeeze


def device_status(raise_on_error=True):
    """Synchronise the current stream and read/clear the device status bits."""
    flags = ctypes.c_uint32(0)
    rc = lib().mv_device_status(_stream(), ctypes.byref(flags))
    if rc not in (0, 6):
        check(rc)
    if flags.value and raise_on_error:
        names = [n for b, n in _STATUS_BITS.items() if flags.value & b]
        raise _lib.MatvansError(6, "device checks failed: " + ", ".join(names))
    return flags.value


class _Matrix:
    rows: int
    cols: int

    def matvec(self, x, scales=None, out=None, out_scaled=None, tuning=None):
        x2, squeeze = _as_x(x, self.cols, self.device)
        B = x2.shape[0]
        y = out if out is not None else torch.empty((B, self.rows), dtype=torch.int32, device=self.device)
        ys = None
        if scales is not None:
            scales = scales if isinstance(scales, torch.Tensor) else torch.from_numpy(np.asarray(scales, np.float32))
            scales = scales.to(self.device, torch.float32).contiguous()
            ys = out_scaled if out_scaled is not None else torch.empty((B, self.rows), dtype=torch.float32,
                                                                      device=self.device)
        if tuning is not None:
            self._launch_tuned(x2, B, y, scales, ys, tuning)
        else:
            self._launch(x2, B, y, scales, ys)
        if squeeze:
            return (y[0], ys[0]) if ys is not None else y[0]
        return (y, ys) if ys is not None else y


class AwrMatrix(_Matrix):
    """A matrix in the reference's ans-warp-rows layout (buffered/encoder.py:394-461)."""

    def __init__(self, compressed, warp_offsets, ppf, ppf_cum, ppf_prob, rows, cols, device="cuda"):
        self.device = torch.device(device)
        self.rows, self.cols = int(rows), int(cols)
        self.compressed = _dev(np.asarray(compressed, np.uint32), self.device)
        self.offsets = _dev(np.asarray(warp_offsets, np.uint32), self.device)
        self.ppf = _dev(np.asarray(ppf, np.uint32), self.device)
        self.ppf_cum = _dev(np.asarray(ppf_cum, np.uint32), self.device)
        self.ppf_prob = _dev(np.asarray(ppf_prob, np.uint32), self.device)
        self.n_words = int(np.asarray(compressed).size)

    @classmethod
    def encode(cls, W, device="cuda"):
        from . import codec
        comp, offs, mn, cdf = codec.compress_ans_warp_rows(W, 32)
        p, pc, pp = codec.decoder_model_from_128bit_encoder_model(mn, cdf)
        return cls(comp, offs, codec.pack_4bytes(p), codec.pack_4bytes(pc), codec.pack_4bytes(pp),
                   W.shape[0], W.shape[1], device)

    @property
    def payload_bytes(self):
        return 4 * self.n_words + 4 * self.rows + 3 * 128

    def _launch(self, x2, B, y, scales, ys):
        check(lib().mv_awr_matvec(_p(self.compressed), self.n_words, _p(self.offsets), _p(self.ppf),
                                  _p(self.ppf_cum), _p(self.ppf_prob), self.rows, self.cols, _p(x2), B, _p(y),
                                  _p(scales), _p(ys), _stream()))

    def matvec_requant(self, x, scale, out=None):
        """Fused int8 output of ans-warp-rows-kernel.cu:212-220."""
        x2, _ = _as_x(x, self.cols, self.device)
        out = out if out is not None else torch.empty(self.rows, dtype=torch.int8, device=self.device)
        check(lib().mv_awr_matvec_requant(_p(self.compressed), self.n_words, _p(self.offsets), _p(self.ppf),
                                          _p(self.ppf_cum), _p(self.ppf_prob), self.rows, self.cols, _p(x2),
                                          ctypes.c_float(scale), _p(out), _stream()))
        return out


class AwsMatrix(AwrMatrix):
    """A matrix in the reference's ans-warp-stripes layout (buffered/encoder.py:323-391): the AWR coder
    and tables, one warp per 32-row stripe, one offset per stripe."""

    @classmethod
    def encode(cls, W, device="cuda"):
        from . import codec
        comp, offs, mn, cdf = codec.compress_ans_warp_stripes(W, 32)
        p, pc, pp = codec.decoder_model_from_128bit_encoder_model(mn, cdf)
        return cls(comp, offs, codec.pack_4bytes(p), codec.pack_4bytes(pc), codec.pack_4bytes(pp),
                   W.shape[0], W.shape[1], device)

    @property
    def payload_bytes(self):
        return 4 * self.n_words + 4 * (self.rows // 32) + 3 * 128

    def _launch(self, x2, B, y, scales, ys):
        check(lib().mv_aws_matvec(_p(self.compressed), self.n_words, _p(self.offsets), _p(self.ppf),
                                  _p(self.ppf_cum), _p(self.ppf_prob), self.rows, self.cols, _p(x2), B, _p(y),
                                  _p(scales), _p(ys), _stream()))

    def matvec_requant(self, x, scale, out=None):
        """Fused int8 output of ans-warp-stripes-kernel.cu:220-226."""
        x2, _ = _as_x(x, self.cols, self.device)
        out = out if out is not None else torch.empty(self.rows, dtype=torch.int8, device=self.device)
        check(lib().mv_aws_matvec_requant(_p(self.compressed), self.n_words, _p(self.offsets), _p(self.ppf),
                                          _p(self.ppf_cum), _p(self.ppf_prob), self.rows, self.cols, _p(x2),
                                          ctypes.c_float(scale), _p(out), _stream()))
        return out


class WprMatrix(_Matrix):
    """A matrix in the reference's matvansWarpPerRow .bin layout."""

    def __init__(self, cm, device="cuda"):
        self.device = torch.device(device)
        self.rows, self.cols = cm.rows, cm.cols
        self.min_value, self.G = int(cm.min_value), int(len(cm.cdf) - 1)
        self.payload_size = int(len(cm.payload))
        pay = np.zeros(self.payload_size + 8, np.uint16)  # keep the tail 16-byte readable
        pay[:self.payload_size] = cm.payload
        self.payload = _dev(pay, self.device)
        self.cursors = _dev(np.asarray(cm.cursors, np.uint32), self.device)
        self.cdf = _dev(np.asarray(cm.cdf, np.uint8), self.device)
        self.ppf = _dev(np.asarray(cm.ppf, np.uint8), self.device)

    @classmethod
    def encode(cls, W, device="cuda"):
        from . import codec
        return cls(codec.encode_matrix(W), device)

    @property
    def payload_bytes(self):
        return 2 * self.payload_size + 4 * self.rows + 256 + self.G + 1

    def _launch(self, x2, B, y, scales, ys):
        check(lib().mv_wpr_matvec(_p(self.payload), self.payload_size, _p(self.cursors),
                                  ctypes.c_int8(self.min_value), _p(self.cdf), self.G, _p(self.ppf), self.rows,
                                  self.cols, _p(x2), B, _p(y), _p(scales), _p(ys), _stream()))


class Q8Matrix(_Matrix):
    """A matrix in this library's Q8-stripe layout (global or per-row tables)."""

    def __init__(self, enc, device="cuda"):
        self.device = torch.device(device)
        self.rows, self.cols = int(enc["rows"]), int(enc["cols"])
        self.blocks = _dev(enc["blocks"], self.device)
        self.blk_off = _dev(enc["blk_off"], self.device)
        self.tbl = _dev(np.asarray(enc["tbl"], np.uint16).view(np.int16), self.device)
        self.tbl_off = _dev(enc["tbl_off"], self.device)
        self.seg_quads, self.nseg = int(enc["seg_quads"]), int(enc["nseg"])
        self.local, self.max_blk_rows = int(enc["local"]), int(enc["max_blk_rows"])
        self.tbl_stripe_max = int(enc["tbl_stripe_max"])
        self.payload_bytes = int(enc["payload_bytes"])
        self.bits_per_weight = float(enc["bits_per_weight"])
        self._view = self.view()

    @classmethod
    def encode(cls, W, local=True, seg_quads=0, device="cuda"):
        from . import codec
        return cls(codec.q8_encode(W, local=local, seg_quads=seg_quads), device)

    def to_encoding(self):
        """The host form of this matrix (q8_encode's dict), e.g. for codec.save_q8."""
        e = {"rows": self.rows, "cols": self.cols, "seg_quads": self.seg_quads, "nseg": self.nseg,
             "local": self.local, "max_blk_rows": self.max_blk_rows, "tbl_stripe_max": self.tbl_stripe_max,
             "payload_bytes": self.payload_bytes, "bits_per_weight": self.bits_per_weight}
        e["blocks"] = self.blocks.cpu().numpy().view(np.uint32)
        e["blk_off"] = self.blk_off.cpu().numpy().view(np.uint32)
        e["tbl"] = self.tbl.cpu().numpy().view(np.uint16)
        e["tbl_off"] = self.tbl_off.cpu().numpy().view(np.uint32)
        return e

    def view(self):
        return Q8View(self.blocks.data_ptr(), self.blk_off.data_ptr(), self.tbl.data_ptr(),
                      self.tbl_off.data_ptr(), self.rows, self.cols, self.seg_quads, self.nseg, self.local,
                      self.max_blk_rows, self.blocks.numel() // 32, self.tbl.numel(), self.tbl_stripe_max)

    def _launch(self, x2, B, y, scales, ys):
        check(lib().mv_q8_matvec(ctypes.byref(self._view), _p(x2), B, _p(y), _p(scales), _p(ys), _stream()))

    def _launch_tuned(self, x2, B, y, scales, ys, tuning):
        t = tuning if isinstance(tuning, Q8Tuning) else Q8Tuning(*tuning)
        check(lib().mv_q8_matvec_tuned(ctypes.byref(self._view), _p(x2), B, _p(y), _p(scales), _p(ys),
                                       ctypes.byref(t), _stream()))

    def _tuning_ptr(self, tuning):
        if tuning is None:
            return None
        t = tuning if isinstance(tuning, Q8Tuning) else Q8Tuning(*tuning)
        self._last_tuning = t
        return ctypes.byref(t)

    def matvec_bf16(self, x, scales, out=None, tuning=None):
        """Float form y = diag(scales) W x: x bf16 [B, cols] -> fp32 [B, rows]."""
        x2 = x.reshape(1, -1) if x.dim() == 1 else x
        if x2.dtype != torch.bfloat16 or x2.shape[-1] != self.cols:
            raise ValueError(f"x must be bf16 with {self.cols} columns")
        x2 = x2.to(self.device).contiguous()
        s = scales.to(self.device, torch.float32).contiguous()
        y = out if out is not None else torch.empty((x2.shape[0], self.rows), dtype=torch.float32, device=self.device)
        check(lib().mv_q8_matvec_bf16(ctypes.byref(self._view), _p(x2), x2.shape[0], _p(s), _p(y),
                                      self._tuning_ptr(tuning), _stream()))
        return y[0] if x.dim() == 1 else y

    def matvec_t_bf16(self, dy, scales, out=None, tuning=None):
        """Transposed float form dx = W^T (scales * dy): dy bf16 [B, rows] -> fp32 [B, cols],
        re-decoding the streams."""
        d2 = dy.reshape(1, -1) if dy.dim() == 1 else dy
        if d2.dtype != torch.bfloat16 or d2.shape[-1] != self.rows:
            raise ValueError(f"dy must be bf16 with {self.rows} columns")
        d2 = d2.to(self.device).contiguous()
        s = scales.to(self.device, torch.float32).contiguous()
        dx = out if out is not None else torch.empty((d2.shape[0], self.cols), dtype=torch.float32, device=self.device)
        check(lib().mv_q8_matvec_t_bf16(ctypes.byref(self._view), _p(d2), d2.shape[0], _p(s), _p(dx),
                                        self._tuning_ptr(tuning), _stream()))
        return dx[0] if dy.dim() == 1 else dx

    def decode(self):
        W = torch.empty((self.rows, self.cols), dtype=torch.int8, device=self.device)
        check(lib().mv_q8_decode(ctypes.byref(self._view), _p(W), _stream()))
        return W


def load_q8(path, device="cuda"):
    """Every matrix of a Q8 file (codec.save_q8 / mv_q8_save) on `device`: (matrices, row_scales, chain) with
    row_scales a list of fp32 device tensors (None where the file has none) and chain the file's chain data
    (host arrays, None when absent)."""
    from . import codec
    encs, scales, chain = codec.load_q8(path)
    dev = torch.device(device)
    mats = [Q8Matrix(e, dev) for e in encs]
    return mats, [None if s is None else torch.from_numpy(s).to(dev) for s in scales], chain


class Q8Stack:
    """Many Q8 matrices (uneven shapes) with their inputs and outputs, run by ONE
    persistent launch (mv_q8_stack_matvec).  Inputs x_i [batch, cols_i] and
    outputs y_i [batch, rows_i] are fixed device tensors, so run() can be
    captured in a CUDA graph and replayed."""

    def __init__(self, matrices, batch=1, tuning=None, xs=None, scales=None, device="cuda"):
        self.device = torch.device(device)
        self.matrices = list(matrices)
        self.batch = int(batch)
        if not 1 <= self.batch <= 16:
            raise ValueError("batch must be 1..16")
        self.tuning = tuning if isinstance(tuning, Q8Tuning) else Q8Tuning(*(tuning or (0, 0, 0, 0)))
        self.xs = xs if xs is not None else [torch.zeros((self.batch, M.cols), dtype=torch.int8, device=self.device)
                                             for M in self.matrices]
        # outputs: views into one contiguous int32 buffer in job order (y_flat), so that one copy moves them all
        sizes = [self.batch * M.rows for M in self.matrices]
        self.y_flat = torch.empty(sum(sizes), dtype=torch.int32, device=self.device)
        self.ys = [v.view(self.batch, M.rows) for v, M in zip(torch.split(self.y_flat, sizes), self.matrices)]
        self.scales = scales
        self.yss = [torch.empty((self.batch, M.rows), dtype=torch.float32, device=self.device)
                    for M in self.matrices] if scales is not None else None
        n = len(self.matrices)
        jobs = (Q8Job * n)()
        # 3..16 vectors run on the tensor cores (engine 0): x is laid out in tiles first (device scratch per
        # matrix)
        self._tiled = self.batch >= MMA_MIN_BATCH and self.tuning.engine == 0
        use_tiles = self._tiled
        self.x_tiles = []
        for i, M in enumerate(self.matrices):
            x = self.xs[i]
            if x.dtype != torch.int8 or tuple(x.shape) != (self.batch, M.cols) or not x.is_contiguous():
                raise ValueError(f"x[{i}] must be a contiguous int8 tensor of shape {(self.batch, M.cols)}")
            jobs[i].m = M.view()
            jobs[i].x = x.data_ptr()
            jobs[i].y = self.ys[i].data_ptr()
            if use_tiles:
                nb = lib().mv_q8_x_tiles_bytes(ctypes.byref(jobs[i].m))
                t = torch.empty(nb, dtype=torch.uint8, device=self.device)
                self.x_tiles.append(t)
                jobs[i].x_tiles = t.data_ptr()
            if scales is not None:
                jobs[i].scales = scales[i].data_ptr()
                jobs[i].ys = self.yss[i].data_ptr()
        self.info = Q8StackInfo()
        check(lib().mv_q8_stack_plan(jobs, n, ctypes.byref(self.tuning), ctypes.byref(self.info)))
        raw = np.frombuffer(bytes(jobs), dtype=np.uint8)
        self.jobs_dev = torch.from_numpy(raw.copy()).to(self.device)
        self._jobs_host = jobs

    @property
    def nitems(self):
        return self.info.nitems

    @property
    def launches_per_run(self):
        """Kernels one run() launches: the persistent decode, the x-tile layout pass when the tensor-core
        consumer reads x tiles, and the zero/scale passes when any job accumulates atomically."""
        return 1 + (1 if self._tiled else 0) + (2 if self.info.atomic_jobs else 0)

    def run(self):
        check(lib().mv_q8_stack_matvec(_p(self.jobs_dev), len(self.matrices), ctypes.byref(self.info), self.batch,
                                       ctypes.byref(self.tuning), _stream()))
        return self.ys


class Q8Chain:
    """A chain of Q8 matrices run as the reference's end-to-end workload
    (buffered/ans-warp-rows.cu:208-221): x_{j+1} = clamp(round(y_j * scale_j), -128, 127),
    with y_j = W_j x_j, every step in ONE persistent, cooperative launch
    (mv_q8_chain_matvec).  rows of matrix j must equal cols of matrix j+1.
    After run(): xs[j] holds matrix j's input (xs[0] the given one), ys[j] its int32
    output, out8 the final int8 vector(s) [batch, rows_last]."""

    def __init__(self, matrices, scales, batch=1, tuning=None, x0=None, device="cuda"):
        self.device = torch.device(device)
        self.matrices = list(matrices)
        self.batch = int(batch)
        if not 1 <= self.batch <= 16:
            raise ValueError("batch must be 1..16")
        if len(scales) != len(self.matrices):
            raise ValueError("one scale per matrix")
        # a chain launch is cooperative (one CTA per SM on the tensor cores) and each step's work items are
        # whole stripes: 16-warp CTAs give each stripe the most warps
        default = (16, 1, 1, 0)
        self.tuning = tuning if isinstance(tuning, Q8Tuning) else Q8Tuning(*(tuning or default))
        self.scales = torch.tensor([float(s) for s in scales], dtype=torch.float32, device=self.device)
        self.xs = [x0 if x0 is not None else torch.zeros((self.batch, self.matrices[0].cols), dtype=torch.int8,
                                                          device=self.device)]
        self.xs += [torch.zeros((self.batch, M.cols), dtype=torch.int8, device=self.device)
                    for M in self.matrices[1:]]
        # outputs: views into one contiguous int32 buffer in job order (y_flat), so that one copy moves them all
        sizes = [self.batch * M.rows for M in self.matrices]
        self.y_flat = torch.empty(sum(sizes), dtype=torch.int32, device=self.device)
        self.ys = [v.view(self.batch, M.rows) for v, M in zip(torch.split(self.y_flat, sizes), self.matrices)]
        self.out8 = torch.empty((self.batch, self.matrices[-1].rows), dtype=torch.int8, device=self.device)
        n = len(self.matrices)
        jobs = (Q8Job * n)()
        for i, M in enumerate(self.matrices):
            x = self.xs[i]
            if x.dtype != torch.int8 or tuple(x.shape) != (self.batch, M.cols) or not x.is_contiguous():
                raise ValueError(f"x[{i}] must be a contiguous int8 tensor of shape {(self.batch, M.cols)}")
            jobs[i].m = M.view()
            jobs[i].x = x.data_ptr()
            jobs[i].y = self.ys[i].data_ptr()
        self.info = Q8StackInfo()
        check(lib().mv_q8_chain_plan(jobs, n, ctypes.byref(self.tuning), ctypes.byref(self.info)))
        raw = np.frombuffer(bytes(jobs), dtype=np.uint8)
        self.jobs_dev = torch.from_numpy(raw.copy()).to(self.device)

    def run(self):
        check(lib().mv_q8_chain_matvec(_p(self.jobs_dev), len(self.matrices), ctypes.byref(self.info), self.batch,
                                       _p(self.scales), _p(self.out8), ctypes.byref(self.tuning), _stream()))
        return self.out8


def dense_matvec(W, x, out=None):
    """Dense int8 comparator y = W x on the GPU (W [rows, cols] int8 device tensor)."""
    rows, cols = W.shape
    x2, squeeze = _as_x(x, cols, W.device)
    y = out if out is not None else torch.empty((x2.shape[0], rows), dtype=torch.int32, device=W.device)
    check(lib().mv_dense_matvec(_p(W), rows, cols, _p(x2), x2.shape[0], _p(y), _stream()))
    return y[0] if squeeze else y


def mat_vec_mul_coalesced(in_vector_gpu, out_vector_gpu, in_dim, out_dim, scale, compressed, warp_offsets, ppf,
                          ppf_cum, ppf_prob):
    """The reference launcher of buffered/ans-warp-rows.cu:38-60, on torch device tensors
    (legacy default stream, like the reference)."""
    lib().mat_vec_mul_coalesced(_p(in_vector_gpu), _p(out_vector_gpu), int(in_dim), int(out_dim),
                                ctypes.c_float(scale), _p(compressed), _p(warp_offsets), _p(ppf), _p(ppf_cum),
                                _p(ppf_prob))
    err = lib().mv_last_error().decode()
    return err


def mat_vec_mul_coalesced_stripes(in_vector_gpu, out_vector_gpu, in_dim, out_dim, scale, compressed, warp_offsets,
                                  ppf, ppf_cum, ppf_prob):
    """The reference launcher of buffered/ans-warp-stripes.cu:38-60 (renamed: the rows program uses the
    same name), on torch device tensors, legacy default stream."""
    lib().mat_vec_mul_coalesced_stripes(_p(in_vector_gpu), _p(out_vector_gpu), int(in_dim), int(out_dim),
                                        ctypes.c_float(scale), _p(compressed), _p(warp_offsets), _p(ppf),
                                        _p(ppf_cum), _p(ppf_prob))
    return lib().mv_last_error().decode()


def requant_absmax(y, out8=None):
    """Fused epilogue of matvansWarpPerRow.cu:51-72,167-172: returns (int8 vector, delta tensor)."""
    n = y.numel()
    out8 = out8 if out8 is not None else torch.empty(n, dtype=torch.int8, device=y.device)
    delta = torch.empty(1, dtype=torch.float32, device=y.device)
    scratch = torch.empty(1, dtype=torch.int32, device=y.device)
    check(lib().mv_requant_absmax(_p(y), n, _p(out8), _p(delta), _p(scratch), _stream()))
    return out8, delta
