"""GPU parity of the batching form (cg3mBatchPlan*): one persistent launch over
a heterogeneous list of problems.

1. Every output is bit-identical to the oracle's model of the plain FP32 3M
   arithmetic with the K split the plan reports (oracle_cgemm3m_fp32), on a
   mixed list: all 16 op pairs (R included), ragged sizes around the tile
   edges, padded leading dimensions (padding left untouched), alpha = 0 and
   k = 0 (beta-only; checked against the reference-order cgemm), quick returns
   (m = 0, alpha = 0 with beta = 1), unit alpha/beta, and forced K splits.
2. The 512-problem heterogeneous workload (m, n, k log-uniform in [16, 1024],
   9 op pairs, random alpha/beta) equals, byte for byte, 512 separate
   cg3mCgemm3mEx calls with the same K split; graph replay and direct launch
   agree; a second replay from the same C gives the same bytes.
"""
import numpy as np
import pytest

from gpu_util import same_bits, to_dev, to_host

pytestmark = pytest.mark.gpu

OPS4 = ["N", "T", "C", "R"]


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _span(k, parts):
    """kSpan = ceil(ceil(k/16)/parts)*16 (the whole K when unsplit)."""
    if parts <= 1:
        return k
    blocks = (k + 15) // 16
    return (blocks + parts - 1) // parts * 16


def _host_problems(oracle):
    rng = np.random.default_rng(99)
    shapes = []
    for i, (ta, tb) in enumerate([(a, b) for a in OPS4 for b in OPS4]):
        m = int(rng.choice([1, 15, 16, 17, 31, 33, 63, 65, 100, 129]))
        n = int(rng.choice([1, 15, 16, 17, 31, 33, 63, 65, 100]))
        k = int(rng.choice([1, 7, 16, 17, 64, 100, 255]))
        shapes.append((ta, tb, m, n, k, complex(0.75, -0.5), complex(0.5, 0.25), i % 3))
    shapes += [
        ("N", "N", 40, 40, 2000, complex(1, 0), complex(0, 0), 0),   # long K: split
        ("C", "T", 130, 70, 1500, complex(0.3, 0.9), complex(-0.2, 0.1), 5),
        ("T", "R", 64, 64, 64, complex(1, 0), complex(0, 0), 0),     # unit
        ("N", "C", 50, 30, 40, complex(0, 0), complex(0.5, -1.5), 3),  # alpha = 0: beta only
        ("T", "N", 20, 25, 0, complex(2, 1), complex(0.25, 0.5), 1),   # k = 0: beta only
        ("N", "N", 0, 10, 10, complex(1, 0), complex(1, 0), 0),        # m = 0: quick return
        ("N", "T", 12, 13, 14, complex(0, 0), complex(1, 0), 2),       # alpha = 0, beta = 1: quick return
        ("R", "C", 200, 150, 300, complex(-1, 0.5), complex(0, 0), 7),
    ]
    probs = []
    for s, (ta, tb, m, n, k, alpha, beta, pad) in enumerate(shapes):
        ar, ac = oracle.stored_shape(ta, m, k)
        br, bc = oracle.stored_shape(tb, k, n)
        lda, ldb, ldc = max(1, ar + pad), max(1, br + pad), max(1, m + pad)
        a = oracle.make_matrix(ar, ac, lda, "RANDOM_NORM_5_5", 1000 + 3 * s)
        b = oracle.make_matrix(br, bc, ldb, "RANDOM_NORM_5_5", 1001 + 3 * s)
        c = oracle.make_matrix(m, n, ldc, "RANDOM_NORM_5_5", 1002 + 3 * s)
        probs.append((ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc))
    return probs


@pytest.mark.parametrize("tune", [False, True])
def test_batch_bit_exact_vs_model(cg3m, oracle, cuda, h, tune):
    import torch

    host = _host_problems(oracle)
    dev = [(ta, tb, m, n, k, al, to_dev(a, torch, cuda), lda, to_dev(b, torch, cuda), ldb, be,
            to_dev(c, torch, cuda), ldc) for (ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc) in host]
    plan = h.batch_plan(dev, tune=tune)
    desc = plan.describe()
    assert any(kp > 1 for _, _, kp in desc), "the long-K problems must be split"
    plan.execute(use_graph=True)
    torch.cuda.synchronize()
    for i, ((ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc), d) in enumerate(zip(host, dev)):
        out = to_host(d[11])
        model = c.copy()
        if m == 0 or n == 0 or ((al == 0 or k == 0) and be == 1):
            assert desc[i] == (0, 0, 0)
        elif al == 0 or k == 0:
            oracle.cgemm(ta, tb, m, n, k, al, a, lda, b, ldb, be, model, ldc)
        else:
            oracle.cgemm3m_fp32_model(ta, tb, m, n, k, al, a, lda, b, ldb, be, model, ldc,
                                      span=_span(k, desc[i][2]))
        assert same_bits(out, model), (i, ta, tb, m, n, k, desc[i])
    plan.close()


def test_batch_512_equals_separate_calls(cg3m, cuda, h):
    import torch
    from cg3m.workloads import batch_problems

    probs = batch_problems(cuda, count=512)
    c0 = [p[11].clone() for p in probs]
    plan = h.batch_plan(probs, tune=True)
    desc = plan.describe()
    plan.execute(use_graph=True)
    torch.cuda.synchronize()
    batch_out = [p[11].clone() for p in probs]
    # replay from the same C: same bytes; direct launch: same bytes
    for use_graph in (True, False):
        for p, c in zip(probs, c0):
            p[11].copy_(c)
        plan.execute(use_graph=use_graph)
        torch.cuda.synchronize()
        for p, ref in zip(probs, batch_out):
            assert torch.equal(p[11].view(torch.float32), ref.view(torch.float32))
    # separate drop-in calls with the plan's K split
    worst = 0.0
    for i, ((ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc), c, (tm, tn, kp)) in enumerate(zip(probs, c0, desc)):
        C2 = c.clone()
        info = h.cgemm3m(ta, tb, m, n, k, al, A, lda, B, ldb, be, C2, ldc, form="fp32", rounding="off",
                         k_partitions=kp)
        assert info["k_partitions"] == kp
        torch.cuda.synchronize()
        assert torch.equal(C2.view(torch.float32), batch_out[i].view(torch.float32)), (i, ta, tb, m, n, k, kp)
        if i % 64 == 0:
            # sanity: normwise error against complex128
            def op(X, o, r, cc):
                M = X.view(cc, r).T.to(torch.complex128)
                return {"N": M, "T": M.T, "C": M.conj().T}[o]
            ar, ac = (m, k) if ta == "N" else (k, m)
            br, bc = (k, n) if tb == "N" else (n, k)
            Z = al * (op(A, ta, ar, ac) @ op(B, tb, br, bc)) + be * c.view(n, m).T.to(torch.complex128)
            got = batch_out[i].view(n, m).T.to(torch.complex128)
            err = (torch.linalg.norm(got - Z) / torch.linalg.norm(Z)).item()
            worst = max(worst, err)
    assert worst < 1e-5
    plan.close()
