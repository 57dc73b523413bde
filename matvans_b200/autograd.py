"""Differentiable float form of the entropy-coded matvec.

y = diag(s) . W_q . x for BF16 activations x [B, cols] with FP32 accumulation,
where W_q is an int8 matrix stored as Q8-stripe rANS streams.  The backward
pass computes dx = W_q^T (s . dy) by decoding the streams again (W_q is never
materialised, neither in the forward nor in the backward), with dy rounded to
BF16 as the kernel consumes it.  W_q and s are constants (no gradient).
"""
import torch

from .ops import Q8Matrix


class Q8LinearFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, matrix, scales):
        ctx.matrix = matrix
        ctx.save_for_backward(scales)
        ctx.x_dtype = x.dtype
        return matrix.matvec_bf16(x.to(torch.bfloat16), scales)

    @staticmethod
    def backward(ctx, gy):
        (scales,) = ctx.saved_tensors
        dx = ctx.matrix.matvec_t_bf16(gy.to(torch.bfloat16).contiguous(), scales)
        return dx.to(ctx.x_dtype), None, None


def q8_linear(x, matrix, scales):
    """Functional form: fp32 [B, rows] = diag(scales) W x for bf16 x [B, cols]."""
    return Q8LinearFunction.apply(x, matrix, scales)


class Q8Linear(torch.nn.Module):
    """A frozen int8 linear layer whose weights live only as rANS streams."""

    def __init__(self, W_q, scales, local=True, device="cuda"):
        super().__init__()
        import numpy as np
        self.matrix = Q8Matrix.encode(np.ascontiguousarray(W_q, dtype=np.int8), local=local, device=device)
        self.register_buffer("scales", torch.as_tensor(scales, dtype=torch.float32, device=device))

    @property
    def in_features(self):
        return self.matrix.cols

    @property
    def out_features(self):
        return self.matrix.rows

    def forward(self, x):
        return q8_linear(x, self.matrix, self.scales)
