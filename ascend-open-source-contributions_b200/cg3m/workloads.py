"""Seeded synthetic workloads on the device.

``batch_problems`` draws the heterogeneous batch: ``count`` independent
problems with m, n, k log-uniform integers in [lo, hi], ops uniform over the 9
(N, T, C) pairs, entries iid complex Uniform(-1, 1), alpha and beta complex with
modulus <= 1 (uniform radius and angle), column-major with ld = stored rows.
"""
from __future__ import annotations

import math

import numpy as np

OPS3 = ("N", "T", "C")


def stored_shape(op, rows_of_op, cols_of_op):
    return (rows_of_op, cols_of_op) if op in ("N", "R") else (cols_of_op, rows_of_op)


def _uniform_complex(n, gen, device):
    import torch

    v = torch.rand(2 * n, generator=gen, device=device, dtype=torch.float32) * 2 - 1
    return torch.view_as_complex(v.view(n, 2))


def batch_shapes(count=512, lo=16, hi=1024, seed=20261029):
    """[(ta, tb, m, n, k, alpha, beta)] of the batch (host side only)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        m, n, k = (int(round(math.exp(x))) for x in rng.uniform(math.log(lo), math.log(hi), 3))
        combo = int(rng.integers(9))
        ta, tb = OPS3[combo // 3], OPS3[combo % 3]
        ra, pa, rb, pb = rng.uniform(0, 1), rng.uniform(0, 2 * math.pi), rng.uniform(0, 1), rng.uniform(0, 2 * math.pi)
        alpha = complex(ra * math.cos(pa), ra * math.sin(pa))
        beta = complex(rb * math.cos(pb), rb * math.sin(pb))
        out.append((ta, tb, m, n, k, alpha, beta))
    return out


def batch_problems(device, count=512, lo=16, hi=1024, seed=20261029):
    """Device buffers for ``batch_shapes``: list of problem tuples
    (ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc) with flat complex64
    tensors (column-major storage)."""
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    probs = []
    for ta, tb, m, n, k, alpha, beta in batch_shapes(count, lo, hi, seed):
        ar, ac = stored_shape(ta, m, k)
        br, bc = stored_shape(tb, k, n)
        A = _uniform_complex(ar * ac, gen, device)
        B = _uniform_complex(br * bc, gen, device)
        C = _uniform_complex(m * n, gen, device)
        probs.append((ta, tb, m, n, k, alpha, A, ar, B, br, beta, C, m))
    return probs


def batch_flops(problems):
    """Sum of 8*m*n*k (complex multiply-add counted as 8 real flops)."""
    return sum(8.0 * p[2] * p[3] * p[4] for p in problems)
