"""The single-phase forward operator as a differentiable torch function.

    y = forward_operator(op, x)            x (K, Ny, Nx) or a batch of slices (B, K, Ny, Nx), CUDA float32
    y.backward(g)  ->  x.grad = A^T g      the hand-written adjoint kernels (op.adjoint_cl), not autograd's tape

The operator is linear, so its vector-Jacobian product is the adjoint itself: SPFO.adjoint_cl (the transposed
pole-figure products, the backprojection with angle weights pi / N_Omega) is the exact transpose of SPFO.direct_cl
(adjoint identity to float32 rounding). With subset=m only the rows of omega subset m are produced (the others are
0) and only those rows reach the gradient. Operators built with pf_mode="generated" recompute their pole-figure
entries in every call instead of storing them, which bounds the memory of a differentiable pipeline; precision="bf16"
operators run both directions through the tensor-core path.

No reference counterpart: diffractom's differentiable module differentiates with respect to model parameters
(differentiable/gradients.py) and has no autograd binding for the coefficients.
"""
from __future__ import annotations

import torch

__all__ = ["SinglePhaseForward", "forward_operator"]


class SinglePhaseForward(torch.autograd.Function):
    """A x with backward A^T g, for one slice (K, Ny, Nx) -> (N_Omega, My, N_eta * N_rings)."""

    @staticmethod
    def forward(ctx, coeffs, op, subset=None):
        x = coeffs.detach().contiguous()
        out = torch.empty(op.data_shape, dtype=torch.float32, device=op.device)
        if subset is not None:
            op._fill(out, 0.0)
        op.direct_cl(x, out, subset=subset)
        ctx.op, ctx.subset = op, subset
        return out

    @staticmethod
    def backward(ctx, grad_out):
        if not ctx.needs_input_grad[0]:
            return None, None, None
        op = ctx.op
        g = grad_out.detach().contiguous()
        if g.dtype != torch.float32:
            g = g.float()
        grad = torch.empty(op.coeff_shape, dtype=torch.float32, device=op.device)
        op.adjoint_cl(g, grad, subset=ctx.subset)
        return grad, None, None


def forward_operator(op, coeffs: torch.Tensor, subset=None) -> torch.Tensor:
    """Differentiable forward model. coeffs: CUDA float32 (K, Ny, Nx) or (B, K, Ny, Nx) (slices projected one after
    the other through the same operator); returns (N_Omega, My, CP) or (B, N_Omega, My, CP). subset: an omega-subset
    index of op.set_omega_subsets (rows of the other angles are 0)."""
    if not isinstance(coeffs, torch.Tensor) or not coeffs.is_cuda or coeffs.dtype != torch.float32:
        raise TypeError("coeffs must be a CUDA float32 tensor")
    shape = tuple(op.coeff_shape)
    if tuple(coeffs.shape) == shape:
        return SinglePhaseForward.apply(coeffs, op, subset)
    if coeffs.dim() == 4 and tuple(coeffs.shape[1:]) == shape:
        return torch.stack([SinglePhaseForward.apply(coeffs[i], op, subset) for i in range(coeffs.shape[0])])
    raise ValueError(f"coeffs must have shape {shape} or (B, *{shape}), not {tuple(coeffs.shape)}")
