"""GPU parity of the plain FP32 3M drop-in (cg3mCgemm3m) against the oracle.

Three bars, as the reference's own test does (ops-blas/test/gemm/cgemm3m/arch35/
cgemm3m_test.cpp:273-308):
  1. the reference accuracy criterion (cgemm3m_verify.h:57-84) against the
     reference-order FP32 cgemm (or FP64 where that is too slow on the host),
     with C padding rows byte-identical;
  2. bitwise determinism: the same call twice gives identical bytes;
  3. additionally, bit-exactness against the oracle's model of this path's
     arithmetic (oracle_cgemm3m_fp32: standard 3M planes, per-partition
     sequential FFMA, fixed-order merge, unrounded-contraction epilogue).
"""
import numpy as np
import pytest

from gpu_util import run, same_bits, sub_problem, to_dev, to_host

pytestmark = pytest.mark.gpu

OPS = ["N", "T", "C"]


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _operands(oracle, ta, tb, m, n, k, pad, fill, seed):
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + pad, br + pad, m + pad
    a = oracle.make_matrix(ar, ac, lda, fill, seed)
    b = oracle.make_matrix(br, bc, ldb, fill, seed + 1)
    c = oracle.make_matrix(m, n, ldc, fill, seed + 2)
    return a, lda, b, ldb, c, ldc


def test_plain_512_exact_and_deterministic(cg3m, oracle, cuda, h):
    import torch

    m = n = k = 512
    alpha, beta = complex(1.5, -0.5), complex(0.25, 0.75)
    a, lda, b, ldb, c, ldc = _operands(oracle, "N", "N", m, n, k, 0, "UNIFORM_1", 20261029)
    out1, info = run(cg3m, h, torch, cuda, "N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    out2, _ = run(cg3m, h, torch, cuda, "N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    assert out1.tobytes() == out2.tobytes(), "identical inputs must give identical bytes"
    model = c.copy()
    oracle.cgemm3m_fp32_model("N", "N", m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
    assert same_bits(out1, model)
    golden = c.copy()
    oracle.cgemm("N", "N", m, n, k, alpha, a, lda, b, ldb, beta, golden, ldc)
    ok, re, im, pad = oracle.verify_cgemm3m(out1, golden, c, m, n, ldc)
    assert ok, (re.__dict__, im.__dict__, pad)
    z = oracle.zgemm_numpy("N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    err = oracle.error_report(oracle.unpack(out1, ldc, m, n), z)
    assert err["normwise"] < 1e-6


@pytest.mark.parametrize("ta", OPS)
@pytest.mark.parametrize("tb", OPS)
def test_nine_ops_padded(cg3m, oracle, cuda, h, ta, tb):
    import torch

    m, n, k = 1000, 777, 3001
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, ta, tb, m, n, k, 13, "UNIFORM_1", 7000 + 3 * OPS.index(ta) +
                                       OPS.index(tb))
    out, info = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    again, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    assert out.tobytes() == again.tobytes()
    z = oracle.zgemm_numpy(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    golden = c.copy()
    golden.reshape(n, ldc)[:, :m] = z.T.astype(np.complex64)
    ok, re, im, pad = oracle.verify_cgemm3m(out, golden, c, m, n, ldc)
    assert ok, (re.__dict__, im.__dict__, pad)
    # bit-exact on a scattered 24 x 20 block of outputs, full K
    rows = np.r_[0:8, 500:508, m - 8:m]
    cols = np.r_[0:7, 388:395, n - 6:n]
    sa, slda = sub_problem(oracle, ta, a, lda, m, k, rows, 0)
    sb, sldb = sub_problem(oracle, tb, b, ldb, k, n, cols, 1)
    sc = np.ascontiguousarray(oracle.unpack(c, ldc, m, n)[np.ix_(rows, cols)].T).reshape(-1)
    oracle.cgemm3m_fp32_model(ta, tb, len(rows), len(cols), k, alpha, sa, slda, sb, sldb, beta, sc, len(rows),
                              span=info["k_span"])
    got = np.ascontiguousarray(oracle.unpack(out, ldc, m, n)[np.ix_(rows, cols)].T).reshape(-1)
    assert same_bits(got, sc)


def test_long_k_split(cg3m, oracle, cuda, h):
    import torch

    m = n = 128
    k = 65536
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, "N", "N", m, n, k, 0, "UNIFORM_1", 4242)
    out, info = run(cg3m, h, torch, cuda, "N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    assert info["k_partitions"] > 1 and info["path"] == 3
    again, _ = run(cg3m, h, torch, cuda, "N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    assert out.tobytes() == again.tobytes()
    z = oracle.zgemm_numpy("N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    golden = z.T.reshape(-1).astype(np.complex64)
    assert oracle.verify_cgemm3m(out, golden, c, m, n, ldc)[0]
    rows = np.r_[0:6, 120:128]
    cols = np.r_[0:5, 60:64, 125:128]
    sa, slda = sub_problem(oracle, "N", a, lda, m, k, rows, 0)
    sb, sldb = sub_problem(oracle, "N", b, ldb, k, n, cols, 1)
    sc = np.ascontiguousarray(oracle.unpack(c, ldc, m, n)[np.ix_(rows, cols)].T).reshape(-1)
    oracle.cgemm3m_fp32_model("N", "N", len(rows), len(cols), k, alpha, sa, slda, sb, sldb, beta, sc, len(rows),
                              span=info["k_span"])
    got = np.ascontiguousarray(oracle.unpack(out, ldc, m, n)[np.ix_(rows, cols)].T).reshape(-1)
    assert same_bits(got, sc)


@pytest.mark.parametrize("parts", [1, 2, 3, 5])
def test_forced_k_partitions_bit_exact(cg3m, oracle, cuda, h, parts):
    import torch

    m, n, k = 70, 45, 999
    alpha, beta = complex(0.3, -1.25), complex(0.5, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, "T", "C", m, n, k, 3, "RANDOM_NORM_5_5", 99 + parts)
    out, info = run(cg3m, h, torch, cuda, "T", "C", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                    k_partitions=parts)
    assert info["k_partitions"] == parts
    model = c.copy()
    oracle.cgemm3m_fp32_model("T", "C", m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
    assert same_bits(out, model)


@pytest.mark.parametrize("parts", [2, 3, 5, 8, 12])
def test_packed_engine_split_merges_bit_exact(cg3m, oracle, cuda, h, parts):
    """The packed engine's K split: 2..8 partitions merge inside the GEMM through
    the tile's cluster (two launches), deeper splits through the merge kernel
    (three); both give the model's bits, on ragged tiles with padded ld."""
    import torch

    m, n, k = 300, 130, 1500
    alpha, beta = complex(0.3, -1.25), complex(0.5, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, "N", "T", m, n, k, 5, "RANDOM_NORM_5_5", 700 + parts)
    out, info = run(cg3m, h, torch, cuda, "N", "T", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                    k_partitions=parts, engine="packed", rounding="off")
    assert info["k_partitions"] == parts and info["path"] == 3
    assert info["kernels"] == (2 if parts <= 8 else 3)
    again, _ = run(cg3m, h, torch, cuda, "N", "T", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                   k_partitions=parts, engine="packed", rounding="off")
    assert out.tobytes() == again.tobytes()
    model = c.copy()
    oracle.cgemm3m_fp32_model("N", "T", m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
    assert same_bits(out, model)


def _fixture_cases(cases, limit=3e6):
    out = []
    for c in cases["cases"]:
        if c["expect"] != "SUCCESS" or c["transa"] == 999 or c["transb"] == 999:
            continue
        if c["m"] * c["n"] * max(c["k"], 1) > limit:
            continue
        if any(f == "NULLPTR" for f in (c["a_fill"], c["b_fill"], c["c_fill"])):
            continue
        out.append(c)
    return out


def test_case_table_rows(cg3m, oracle, cuda, h, cases):
    """Every successful row of the reference's case table up to ~3e6 complex
    multiply-adds: reference criterion vs reference-order cgemm, padding bytes,
    determinism, and bit-exactness vs the model."""
    import torch

    rows = _fixture_cases(cases)
    assert len(rows) > 500
    failures = []
    for cs in rows:
        ta, tb, m, n, k = cs["transa"], cs["transb"], cs["m"], cs["n"], cs["k"]
        ar, ac = oracle.stored_shape(ta, m, k)
        br, bc = oracle.stored_shape(tb, k, n)
        a = oracle.make_matrix(ar, ac, cs["lda"], cs["a_fill"], cs["seed"])
        b = oracle.make_matrix(br, bc, cs["ldb"], cs["b_fill"], cs["seed"] + 1)
        c = oracle.make_matrix(m, n, cs["ldc"], cs["c_fill"], cs["seed"] + 2)
        alpha, beta = complex(*cs["alpha"]), complex(*cs["beta"])
        out, info = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, cs["lda"], b, cs["ldb"], beta, c, cs["ldc"])
        again, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, cs["lda"], b, cs["ldb"], beta, c, cs["ldc"])
        golden = c.copy()
        oracle.cgemm(ta, tb, m, n, k, alpha, a, cs["lda"], b, cs["ldb"], beta, golden, cs["ldc"])
        ok, re, im, pad = oracle.verify_cgemm3m(out, golden, c, m, n, cs["ldc"])
        if not ok:
            failures.append((cs["name"], "criterion", re.__dict__, im.__dict__, pad))
        if not same_bits(out, again):
            failures.append((cs["name"], "nondeterministic"))
        if m and n and k and (alpha != 0):
            model = c.copy()
            oracle.cgemm3m_fp32_model(ta, tb, m, n, k, alpha, a, cs["lda"], b, cs["ldb"], beta, model, cs["ldc"],
                                      span=info["k_span"])
            if not same_bits(out, model):
                failures.append((cs["name"], "model"))
    assert not failures, failures[:10]


def test_empty_output_preserves_sentinel(cg3m, cuda, h):
    """cgemm3m_test.cpp:175-187."""
    import torch

    sentinel = np.full(12, complex(7.0, -3.0), np.complex64)
    for m, n in ((0, 3), (3, 0)):
        C = to_dev(sentinel, torch, cuda)
        st = h.cgemm3m("N", "N", m, n, 2, 1.0, None, 4, None, 4, 0.0, C, 4, raw=True)
        torch.cuda.synchronize()
        assert st == cg3m.SUCCESS
        assert to_host(C).tobytes() == sentinel.tobytes()


def test_zero_product_allows_null_inputs(cg3m, oracle, cuda, h):
    """cgemm3m_test.cpp:189-210: k==0 or alpha==0 with null A/B; beta in
    {0, 1, 0.5-0.25i}; NaN in C is not read when beta==0."""
    import torch

    m, n, ldc = 3, 2, 5
    for zero_k in (True, False):
        k = 0 if zero_k else 7
        alpha = 1.0 if zero_k else 0.0
        for beta in (0j, 1 + 0j, complex(0.5, -0.25)):
            val = complex(np.nan, -3.0) if beta == 0 else complex(7.0, -3.0)
            init = np.full(ldc * n, val, np.complex64)
            C = to_dev(init, torch, cuda)
            st = h.cgemm3m("N", "N", m, n, k, alpha, None, 3, None, 7, beta, C, ldc, raw=True)
            torch.cuda.synchronize()
            assert st == cg3m.SUCCESS
            golden = init.copy()
            oracle.cgemm("N", "N", m, n, k, alpha, None, 3, None, 7, beta, golden, ldc)
            out = to_host(C)
            assert oracle.verify_cgemm3m(out, golden, init, m, n, ldc)[0]


def test_runs_on_caller_stream(cg3m, oracle, cuda):
    import torch

    s = torch.cuda.Stream()
    h = cg3m.Handle(stream=s)
    m, n, k = 200, 150, 300
    a, lda, b, ldb, c, ldc = _operands(oracle, "N", "T", m, n, k, 1, "UNIFORM_1", 5)
    with torch.cuda.stream(s):
        A, B, C = to_dev(a, torch, cuda), to_dev(b, torch, cuda), to_dev(c, torch, cuda)
        info = h.cgemm3m("N", "T", m, n, k, 1.0, A, lda, B, ldb, 0.5, C, ldc)
    s.synchronize()
    model = c.copy()
    oracle.cgemm3m_fp32_model("N", "T", m, n, k, 1.0, a, lda, b, ldb, 0.5, model, ldc, span=info["k_span"])
    assert same_bits(to_host(C), model)
    assert h.device_status() == 0


def test_strided_batched_identity_example(cg3m, cuda):
    """blas/gemm/README.md:854-907: two 2x2 batches with A = I give C = B bitwise."""
    import ctypes

    import torch

    a = np.array([1, 0, 0, 1, 1, 0, 0, 1], np.complex64)
    b = np.array([1, 2, 3, 4, 5, 6, 7, 8], np.complex64)
    A, B = to_dev(a, torch, cuda), to_dev(b, torch, cuda)
    C = torch.zeros(8, dtype=torch.complex64, device=cuda)
    h = cg3m.Handle()
    one, zero = cg3m.cx(1), cg3m.cx(0)
    st = cg3m.lib.cg3mCgemm3mStridedBatched(h.h, 0, 0, 2, 2, 2, ctypes.byref(one), cg3m.ptr(A), 2, 4, cg3m.ptr(B), 2,
                                            4, ctypes.byref(zero), cg3m.ptr(C), 2, 4, 2)
    torch.cuda.synchronize()
    assert st == cg3m.SUCCESS
    assert to_host(C).tobytes() == b.tobytes()
