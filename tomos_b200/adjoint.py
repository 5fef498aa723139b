"""Differentiable least squares over the C ABI.

X = argmin ||A X - B|| column by column (sketch-preconditioned LSQR,
tomos_lsqr_solve_dense), with gradients in A and B from the adjoint:
for a loss L with G = dL/dX,
    Lam   = (A^T A)^{-1} G        (tomos_lsqr_adjoint_batch_dense: all columns at
                                    once, reusing R^{-1})
    dL/dB = A Lam
    dL/dA = (B - A X) Lam^T - (A Lam) X^T
the last two in one pass over A (tomos_lsqr_adjoint_grad_dense).
"""
import torch

from . import (Dense, Layout, NumericType, StopRule, add_precond, apply_count_sketch, column_scale,
               create_lsqr_workspace, generate_sketch_qr_precond, lsqr_adjoint_batch,
               lsqr_adjoint_grad, lsqr_solve)


class LeastSquares(torch.autograd.Function):
    """X = argmin ||A X - B|| for a row-major float32 CUDA A (m x n) and
    B (m x K); differentiable in A and B."""

    @staticmethod
    def forward(ctx, A, B, sketch_rows, tol, max_iters):
        if A.dtype != torch.float32 or not A.is_cuda or A.dim() != 2:
            raise ValueError("lstsq: A must be a 2-D float32 CUDA tensor")
        A = A.contiguous()
        B2 = B.reshape(B.shape[0], -1).contiguous().float()
        m, n = A.shape
        D = Dense(NumericType.FP32, Layout.ROW_MAJOR, (m, n), n, A.view(-1))
        s = sketch_rows or 4 * n
        SA, _, colsq = apply_count_sketch(D, s, with_colsq=True)
        Rinv = generate_sketch_qr_precond(SA)
        dsc, anorm = column_scale(colsq)
        ws = create_lsqr_workspace(None, (m, n), NumericType.FP32, NumericType.FP64)
        add_precond(Rinv, ws)
        X = torch.empty((n, B2.shape[1]), dtype=torch.float32, device=A.device)
        for k in range(B2.shape[1]):
            x = torch.zeros(n, dtype=torch.float32, device=A.device)
            lsqr_solve(None, D, B2[:, k].contiguous(), x, ws, tol, max_iters, 0.0, restarts=4,
                       stop_rule=StopRule.BACKWARD, anorm_fro=anorm, col_scale=dsc)
            X[:, k] = x
        ctx.save_for_backward(A, B2, X)
        ctx.state = (D, ws, Rinv, tol, max_iters, B.shape)
        return X if B.dim() == 2 else X[:, 0]

    @staticmethod
    def backward(ctx, G):
        A, B2, X = ctx.saved_tensors
        D, ws, Rinv, tol, max_iters, bshape = ctx.state
        G2 = G.reshape(X.shape[0], -1).float()
        Lam, _ = lsqr_adjoint_batch(D, G2, ws, tol=min(tol, 1e-7), max_iters=max_iters)
        gA, gB = lsqr_adjoint_grad(D, B2, X, Lam, want_grad_a=ctx.needs_input_grad[0])
        return gA, gB.reshape(bshape), None, None, None


def lstsq(A, B, sketch_rows=None, tol=1e-6, max_iters=200):
    """X = argmin ||A X - B|| (differentiable in A and B)."""
    return LeastSquares.apply(A, B, sketch_rows, tol, max_iters)
