"""The differentiable form: backward through the same 3M kernels via op codes.

CPU: the op-code mapping of both gradients equals torch's complex autograd for
all 16 (opA, opB) pairs (kernel replaced by a complex128 product), and agrees
with central finite differences (h = 1e-3) on scalar projections.
GPU: 16 problems of 1024^3 with random ops plus one 256 x 256 x 65536 problem,
upstream gradient iid complex U(-1,1): the kernels' gradients match a
complex128 torch.matmul reference to 1e-5 relative (normwise), and their
projections match complex128 finite differences to 1e-5 relative.
"""
import itertools

import numpy as np
import pytest
import torch

OPS = "NTCR"


def _op(X, o):
    return {"N": X, "T": X.transpose(-2, -1), "C": X.conj().transpose(-2, -1), "R": X.conj()}[o]


def _shapes(ta, tb, m, n, k):
    sa = (m, k) if ta in "NR" else (k, m)
    sb = (k, n) if tb in "NR" else (n, k)
    return sa, sb


def _uniform(shape, gen, dtype=torch.complex128, device="cpu"):
    re = torch.rand(shape, generator=gen, dtype=torch.float64) * 2 - 1
    im = torch.rand(shape, generator=gen, dtype=torch.float64) * 2 - 1
    return torch.complex(re, im).to(dtype=dtype, device=device)


def test_op_mapping_matches_torch_autograd(cg3m, monkeypatch):
    import cg3m.autograd as ag

    monkeypatch.setattr(ag, "_cgemm3m", lambda X, Y, tx, ty, form=None, rounding=None: _op(X, tx) @ _op(Y, ty))
    gen = torch.Generator().manual_seed(3)
    for ta, tb in itertools.product(OPS, repeat=2):
        sa, sb = _shapes(ta, tb, 5, 4, 6)
        A = _uniform(sa, gen).requires_grad_()
        B = _uniform(sb, gen).requires_grad_()
        dC = _uniform((5, 4), gen)
        gA, gB = torch.autograd.grad(_op(A, ta) @ _op(B, tb), (A, B), dC)
        assert torch.allclose(ag.grad_a(dC, B.detach(), ta, tb), gA, rtol=0, atol=1e-12)
        assert torch.allclose(ag.grad_b(dC, A.detach(), ta, tb), gB, rtol=0, atol=1e-12)


def test_finite_differences_complex128_cpu(cg3m, monkeypatch):
    import cg3m.autograd as ag

    monkeypatch.setattr(ag, "_cgemm3m", lambda X, Y, tx, ty, form=None, rounding=None: _op(X, tx) @ _op(Y, ty))
    gen = torch.Generator().manual_seed(4)
    h = 1e-3
    for ta, tb in (("N", "N"), ("T", "C"), ("C", "R"), ("R", "T")):
        sa, sb = _shapes(ta, tb, 4, 3, 5)
        A, B = _uniform(sa, gen), _uniform(sb, gen)
        W = _uniform((4, 3), gen)
        L = lambda A_, B_: (W.conj() * (_op(A_, ta) @ _op(B_, tb))).sum().real
        gA, gB = ag.grad_a(W, B, ta, tb), ag.grad_b(W, A, ta, tb)
        for which, g in (("A", gA), ("B", gB)):
            V = _uniform(sa if which == "A" else sb, gen)
            if which == "A":
                fd = (L(A + h * V, B) - L(A - h * V, B)) / (2 * h)
            else:
                fd = (L(A, B + h * V) - L(A, B - h * V)) / (2 * h)
            proj = (g.conj() * V).sum().real
            assert abs(fd - proj) <= 1e-9 * max(1.0, abs(fd))


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp32", "tf32x3", "bf16x6"])
def test_gradients_match_complex128_reference(cg3m, cuda, form):
    """16 x 1024^3 with random ops plus 256 x 256 x 65536, forward and backward
    through the same 3M kernels in the given form: gradients within 1e-5 of a
    complex128 reference gradient and of complex128 central differences."""
    from cg3m.autograd import cgemm3m_autograd

    gen = torch.Generator().manual_seed(2026)
    rng = np.random.default_rng(7)
    problems = [(1024, 1024, 1024)] * 16 + [(256, 256, 65536)]
    worst = 0.0
    for (m, n, k) in problems:
        ta, tb = OPS[rng.integers(4)], OPS[rng.integers(4)]
        sa, sb = _shapes(ta, tb, m, n, k)
        A64, B64 = _uniform(sa, gen), _uniform(sb, gen)
        dC64 = _uniform((m, n), gen)
        A = A64.to(torch.complex64).to(cuda).requires_grad_()
        B = B64.to(torch.complex64).to(cuda).requires_grad_()
        out = cgemm3m_autograd(A, B, ta, tb, form)
        out.backward(dC64.to(torch.complex64).to(cuda))
        # complex128 reference gradient from the same complex64 inputs
        Ar = A.detach().to(torch.complex128).requires_grad_()
        Br = B.detach().to(torch.complex128).requires_grad_()
        ref = _op(Ar, ta) @ _op(Br, tb)
        gA, gB = torch.autograd.grad(ref, (Ar, Br), dC64.to(cuda))
        assert torch.linalg.norm(out.detach().to(torch.complex128) - ref.detach()) <= 1e-5 * torch.linalg.norm(ref)
        for g, r in ((A.grad, gA), (B.grad, gB)):
            rel = (torch.linalg.norm(g.to(torch.complex128) - r) / torch.linalg.norm(r)).item()
            worst = max(worst, rel)
            assert rel <= 1e-5, (m, n, k, ta, tb, rel)
        # finite differences (complex128) on a scalar projection L = Re<dC, C>
        h = 1e-3
        V = _uniform(sa, gen).to(cuda)
        L = lambda A_: (dC64.to(cuda).conj() * (_op(A_, ta) @ _op(Br.detach(), tb))).sum().real
        fd = ((L(Ar.detach() + h * V) - L(Ar.detach() - h * V)) / (2 * h)).item()
        proj = (A.grad.to(torch.complex128).conj() * V).sum().real.item()
        assert abs(fd - proj) <= 1e-5 * abs(fd), (fd, proj)
    print(form, "worst relative gradient error", worst)
