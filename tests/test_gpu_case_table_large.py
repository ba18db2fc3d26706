"""The reference's case-table rows above 3e6 complex multiply-adds on the GPU,
through the drop-in exactly as a user calls it (cg3mCgemm3m: the rounding
pass runs where the reference's gate admits the shape).

Per row, as the reference's test does (cgemm3m_test.cpp:273-308): two runs
compared byte for byte, padding rows of C untouched, and the reference
criterion (cgemm3m_verify.h:22-84) -- here on sampled row x column blocks
(first, middle and last rows and columns), whose golden is the reference-order
FP32 cgemm of the oracle on the same rows of op(A) and columns of op(B).  On
those blocks the result must also equal the oracle's bit-exact model: the
plain 3M model, or for the rounding-gated squares (N,N / N,T / T,N / C,C /
C,N orders 2048..4096) the path GEMM's value where unflagged and the
segmented replay where flagged.
"""
import numpy as np
import pytest

from gpu_util import run, same_bits, sub_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _large_rows(cases, limit=3e6):
    out = []
    for c in cases["cases"]:
        if c["expect"] != "SUCCESS" or c["transa"] == 999 or c["transb"] == 999:
            continue
        if any(f == "NULLPTR" for f in (c["a_fill"], c["b_fill"], c["c_fill"])):
            continue
        if c["m"] * c["n"] * max(c["k"], 1) > limit:
            out.append(c)
    return out


def _sample(size, take=32):
    idx = np.r_[0:take, size // 2 - take // 2:size // 2 + take // 2, size - take:size]
    return np.unique(idx[(idx >= 0) & (idx < size)])


def test_case_table_rows_above_3e6(cg3m, oracle, cuda, h, cases):
    import torch

    rows = _large_rows(cases)
    assert len(rows) >= 350
    failures = []
    gated = 0
    for cs in rows:
        ta, tb, m, n, k = cs["transa"], cs["transb"], cs["m"], cs["n"], cs["k"]
        lda, ldb, ldc = cs["lda"], cs["ldb"], cs["ldc"]
        ar, ac = oracle.stored_shape(ta, m, k)
        br, bc = oracle.stored_shape(tb, k, n)
        a = oracle.make_matrix(ar, ac, lda, cs["a_fill"], cs["seed"])
        b = oracle.make_matrix(br, bc, ldb, cs["b_fill"], cs["seed"] + 1)
        c = oracle.make_matrix(m, n, ldc, cs["c_fill"], cs["seed"] + 2)
        alpha, beta = complex(*cs["alpha"]), complex(*cs["beta"])
        out, info = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
        again, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
        if not same_bits(out, again):
            failures.append((cs["name"], "nondeterministic"))
        if ldc > m:
            O = out[: ldc * n].reshape(n, ldc)
            I = c[: ldc * n].reshape(n, ldc)
            if O[:, m:].tobytes() != I[:, m:].tobytes():
                failures.append((cs["name"], "padding written"))
        ri, ci = _sample(m), _sample(n)
        sa, slda = sub_problem(oracle, ta, a, lda, m, k, ri, 0)
        sb, sldb = sub_problem(oracle, tb, b, ldb, k, n, ci, 1)
        init = np.ascontiguousarray(oracle.unpack(c, ldc, m, n)[np.ix_(ri, ci)].T).reshape(-1)
        got = np.ascontiguousarray(oracle.unpack(out, ldc, m, n)[np.ix_(ri, ci)].T).reshape(-1)
        golden = init.copy()
        oracle.cgemm_timing(ta, tb, len(ri), len(ci), k, alpha, sa, slda, sb, sldb, beta, golden, len(ri))
        ok, re, im, _ = oracle.verify_cgemm3m(got, golden, init, len(ri), len(ci), len(ri))
        if not ok:
            failures.append((cs["name"], "criterion", re.__dict__, im.__dict__))
        if alpha == 0 or k == 0:
            continue  # beta-scale only: covered by the criterion above
        if info["rounding"]:
            gated += 1
            e = oracle.energy(m, ta, tb, a, lda, b, ldb)
            path, cpath = oracle.risk_path_rect(len(ri), len(ci), k, ta, sa, slda, tb, sb, sldb)
            P = path.reshape(len(ci), len(ri)).T
            Cm = cpath.reshape(len(ci), len(ri)).T
            flags = oracle.select_flags(P, Cm, e[ri], e[m + ci], oracle.bridge(m))
            opa = oracle.op_matrix(a, lda, ta, m, k)
            opb = oracle.op_matrix(b, ldb, tb, k, n)
            expect = Cm.copy()
            for (r, q) in zip(*np.nonzero(flags)):
                expect[r, q] = oracle.recompute_dot(np.ascontiguousarray(opa[ri[r], :]),
                                                    np.ascontiguousarray(opb[:, ci[q]]))
            model = np.ascontiguousarray(expect.T).reshape(-1).astype(np.complex64)
        else:
            model = init.copy()
            oracle.cgemm3m_fp32_model(ta, tb, len(ri), len(ci), k, alpha, sa, slda, sb, sldb, beta, model, len(ri),
                                      span=info["k_span"])
        if not same_bits(got, model):
            failures.append((cs["name"], "model bits", info))
    assert gated >= 15
    assert not failures, failures[:10]
