"""torch.autograd wrapper of the LU solve and its adjoint, for gradient checking.

X = solve(A, B) factors A with the plain FP64 LU (b2m_dev_MatrixLUDecompInPlace, the reference's
pivots), solves with those factors (b2m_dev_MatrixLUBackSubst), and keeps the factors.  The
backward pass calls the adjoint entry point b2m_dev_MatrixLinEQSolveAdjoint on the same factors:
dB = A^-T dX and dA = -dB X^T.  Everything runs through the C ABI; torch only holds the buffers.
"""
from __future__ import annotations

import torch

from . import linalg as L
from ._lib import Context


class LinEQSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A: torch.Tensor, B: torch.Tensor, bctx: Context | None = None):
        if A.dtype != torch.float64 or B.dtype != torch.float64 or not A.is_cuda:
            raise TypeError("solve: A and B must be float64 CUDA tensors")
        n = A.shape[0]
        LU = A.detach().contiguous().clone()
        indx = torch.zeros(n, dtype=torch.int32, device=A.device)
        status = torch.zeros(1, dtype=torch.int32, device=A.device)
        L.dev_MatrixLUDecompInPlace(LU, indx, status, ctx=bctx)
        X = B.detach().contiguous().clone()
        L.dev_MatrixLUBackSubst(LU, indx, X, ctx=bctx)
        if int(status.item()) != 0:
            raise RuntimeError("solve: singular matrix")
        ctx.save_for_backward(LU, indx, X)
        ctx.bctx = bctx
        return X

    @staticmethod
    def backward(ctx, G: torch.Tensor):
        LU, indx, X = ctx.saved_tensors
        lam = torch.empty_like(X)
        dA = torch.empty_like(LU) if ctx.needs_input_grad[0] else None
        L.dev_MatrixLinEQSolveAdjoint(LU, indx, X, G.contiguous(), lam, dA, ctx=ctx.bctx)
        return dA, (lam if ctx.needs_input_grad[1] else None), None


def solve(A: torch.Tensor, B: torch.Tensor, bctx: Context | None = None) -> torch.Tensor:
    """X = A^-1 B with an autograd backward through the adjoint kernel (B may be 1-D)."""
    squeeze = B.dim() == 1
    X = LinEQSolveFunction.apply(A, B.unsqueeze(1) if squeeze else B, bctx)
    return X.squeeze(1) if squeeze else X
