"""Output-column sharding through the library (cg3m.dist.cgemm3m_local_block),
run rank by rank on one GPU.

The product shards with no exchange (each output column needs all of op(A)
and one column of op(B)); with every rank keeping the whole problem's K
split, the assembled C is the single call's C byte for byte, whatever the
number of ranks -- which is what a G-GPU run relies on.
"""
import numpy as np
import pytest

from gpu_util import to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "T"), ("T", "C")])
@pytest.mark.parametrize("world", [2, 3, 8])
def test_column_blocks_assemble_the_single_call(cg3m, oracle, cuda, ta, tb, world):
    import torch

    from cg3m import dist as cdist

    m, n, k = 700, 523, 900
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + 5, br + 3, m + 7
    a = oracle.make_matrix(ar, ac, lda, "UNIFORM_1", 201)
    b = oracle.make_matrix(br, bc, ldb, "UNIFORM_1", 202)
    c = oracle.make_matrix(m, n, ldc, "UNIFORM_1", 203)
    A, B = to_dev(a, torch, cuda), to_dev(b, torch, cuda)
    h = cg3m.Handle(stream=torch.cuda.current_stream().cuda_stream)
    whole = to_dev(c, torch, cuda)
    info = h.cgemm3m(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, whole, ldc)
    kp = info["k_partitions"]
    sharded = to_dev(c, torch, cuda)
    for rank in range(world):
        cdist.cgemm3m_local_block(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, sharded, ldc, world, rank,
                                  k_partitions=kp)
    torch.cuda.synchronize()
    assert sharded.cpu().numpy().tobytes() == whole.cpu().numpy().tobytes()
    model = c.copy()
    oracle.cgemm3m_fp32_model(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
    assert whole.cpu().numpy().tobytes() == model.tobytes()
