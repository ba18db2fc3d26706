"""Differentiable cgemm3m: ``torch.autograd.Function`` over the 3M kernels.

Semantics on torch (row-major) complex64 matrices: ``out = opt(A) @ opt(B)``
with opt in {N: X, T: X^T, C: X^H, R: conj(X)}, optionally batched over a
leading dimension.  The backward uses PyTorch's convention for complex
matmul (grad_opt(A) = grad_out @ opt(B)^H, grad_opt(B) = opt(A)^H @ grad_out)
and maps each gradient back through opt() by choosing the operand order and
op codes of the same 3M kernels, so no explicit transpose or conjugate is
ever materialised:

    grad A:  N: dC @ H(opt_B)          T: conj(opt_B) @ dC^T
             C: opt_B @ dC^H           R: conj(dC) @ opt_B^T
    grad B:  N: H(opt_A) @ dC          T: dC^T @ conj(opt_A)
             C: dC^H @ opt_A           R: opt_A^T @ conj(dC)

where H/conj/T of an op code compose on its (transpose, conjugate) bits.
"""
from __future__ import annotations

import torch

from . import cgemm3m as _cgemm3m

_BITS = {"N": (0, 0), "T": (1, 0), "C": (1, 1), "R": (0, 1)}
_NAMES = {v: k for k, v in _BITS.items()}


def _h(op):
    t, c = _BITS[op]
    return _NAMES[(t ^ 1, c ^ 1)]


def _conj(op):
    t, c = _BITS[op]
    return _NAMES[(t, c ^ 1)]


def _t(op):
    t, c = _BITS[op]
    return _NAMES[(t ^ 1, c)]


def _mm(X, Y, tx, ty, form):
    """opt(X) @ opt(Y) for 2-D or batched 3-D complex64 tensors."""
    if X.dim() == 2:
        return _cgemm3m(X, Y, tx, ty, form=form, rounding="off")
    return torch.stack([_cgemm3m(X[i], Y[i], tx, ty, form=form, rounding="off") for i in range(X.shape[0])])


def grad_a(dC, B, ta, tb, form="fp32"):
    if ta == "N":
        return _mm(dC, B, "N", _h(tb), form)
    if ta == "T":
        return _mm(B, dC, _conj(tb), "T", form)
    if ta == "C":
        return _mm(B, dC, tb, "C", form)
    return _mm(dC, B, "R", _t(tb), form)


def grad_b(dC, A, ta, tb, form="fp32"):
    if tb == "N":
        return _mm(A, dC, _h(ta), "N", form)
    if tb == "T":
        return _mm(dC, A, "T", _conj(ta), form)
    if tb == "C":
        return _mm(dC, A, "C", ta, form)
    return _mm(A, dC, _t(ta), "R", form)


class Cgemm3mFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, B, transa="N", transb="N", form="fp32"):
        ctx.save_for_backward(A, B)
        ctx.ops = (transa, transb, form)
        return _mm(A.contiguous(), B.contiguous(), transa, transb, form)

    @staticmethod
    def backward(ctx, dC):
        A, B = ctx.saved_tensors
        ta, tb, form = ctx.ops
        dC = dC.contiguous()
        gA = grad_a(dC, B.contiguous(), ta, tb, form) if ctx.needs_input_grad[0] else None
        gB = grad_b(dC, A.contiguous(), ta, tb, form) if ctx.needs_input_grad[1] else None
        return gA, gB, None, None, None


def cgemm3m_autograd(A, B, transa="N", transb="N", form="fp32"):
    """Differentiable ``opt(A) @ opt(B)`` on CUDA complex64 tensors."""
    return Cgemm3mFunction.apply(A, B, transa, transb, form)
