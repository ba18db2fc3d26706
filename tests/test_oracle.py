"""CPU tests of the oracle itself: pinned against the reference's own known
answers before it is trusted as the checker.

Pins used (paths inside the reference's ops-blas/ tree):
  * verifier boundary tests   test/gemm/cgemm3m/arch35/cgemm3m_test.cpp:93-164
  * SegmentCancellation KAT   cgemm3m_test.cpp:212-240
  * ZeroProduct golden        cgemm3m_golden.h:29-45, cgemm3m_test.cpp:189-210
  * case table integrity      cgemm3m_test.cpp:242-267 (1200 rows, 200 TC_PF)
"""
import math

import numpy as np
import pytest


# ---------------------------------------------------------------- verifier KATs

def test_verifier_matched_ratio_and_max_error(oracle):
    r = oracle.Cgemm3mComponentResult()
    for _ in range(99):
        r.add(0.0, 0.0)
    assert r.passed()
    r.add(0.001, 0.0)
    assert r.passed()  # one mismatch among 100 meets 99%
    r.add(0.001, 0.0)
    assert not r.passed()
    for _ in range(99):
        r.add(0.0, 0.0)
    assert r.passed()
    mx = oracle.Cgemm3mComponentResult()
    for _ in range(99):
        mx.add(0.0, 0.0)
    mx.add(0.02, 0.0)
    assert not mx.passed()  # ratio passes, max-error bound fails


def test_verifier_magnitude_scaled_tolerance(oracle):
    r = oracle.Cgemm3mComponentResult()
    r.add(0.001, 0.0)
    assert not r.passed()
    r.add(8192.02, 8192.0)
    assert r.max_error_golden == 8192.0
    assert not r.passed()
    b = oracle.Cgemm3mComponentResult()
    b.add(1.0 / 8192.0, 0.0)
    assert b.passed()
    b.add(2.0 / 8192.0, 0.0)
    assert not b.passed()
    large = oracle.Cgemm3mComponentResult()
    large.add(8192.5, 8192.0)
    assert large.matched == 1
    assert not large.passed()
    ulp = oracle.Cgemm3mComponentResult()
    ulp.add(8192.03125, 8192.0)
    assert ulp.matched == ulp.finite
    assert ulp.passed()
    ulp.add(8192.0625, 8192.0)
    assert ulp.matched == 2
    assert not ulp.passed()


def test_verifier_nonfinite_rules(oracle):
    inf, nan = math.inf, math.nan
    r = oracle.Cgemm3mComponentResult()
    r.add(nan, nan)
    r.add(inf, inf)
    r.add(-inf, -inf)
    assert r.passed()
    for a, g in ((nan, inf), (inf, nan), (-inf, nan), (nan, -inf)):
        e = oracle.Cgemm3mComponentResult()
        e.add(a, g)
        assert e.passed()
    for a, g in ((inf, -inf), (-inf, inf)):
        e = oracle.Cgemm3mComponentResult()
        e.add(a, g)
        assert not e.passed()
    f = oracle.Cgemm3mComponentResult()
    f.add(0.0, inf)
    assert not f.passed()


# ---------------------------------------------------------------- oracle cgemm

OPS = ["N", "T", "C"]


@pytest.mark.parametrize("ta", OPS + ["R"])
@pytest.mark.parametrize("tb", OPS + ["R"])
def test_oracle_cgemm_matches_fp64(oracle, ta, tb):
    m, n, k = 9, 7, 13
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + 3, br + 1, m + 2
    a = oracle.make_matrix(ar, ac, lda, "RANDOM_NORM_5_5", 11)
    b = oracle.make_matrix(br, bc, ldb, "RANDOM_NORM_5_5", 12)
    c = oracle.make_matrix(m, n, ldc, "RANDOM_NORM_5_5", 13)
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    g = c.copy()
    oracle.cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, g, ldc)
    z = oracle.zgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    zn = oracle.zgemm_numpy(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    assert np.abs(z - zn).max() < 1e-9
    got = oracle.unpack(g, ldc, m, n)
    assert np.abs(got - z).max() < 1e-3
    # padding rows untouched, byte for byte
    assert g.reshape(n, ldc)[:, m:].tobytes() == c.reshape(n, ldc)[:, m:].tobytes()
    # the bit-exact 3M model is a valid cgemm under the reference criterion
    x = c.copy()
    oracle.cgemm3m_fp32_model(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, x, ldc, span=5)
    assert oracle.verify_cgemm3m(x, g, c, m, n, ldc)[0]


def test_oracle_zero_product_semantics(oracle):
    """k==0 / alpha==0 golden (cgemm3m_golden.h:29-45): beta==1 leaves C, beta==0
    writes zeros even over NaN, else scales."""
    m, n, ldc = 3, 2, 5
    for beta in (0j, 1 + 0j, complex(0.5, -0.25)):
        init_val = complex(math.nan, -3.0) if beta == 0 else complex(7.0, -3.0)
        c = np.full(ldc * n, init_val, dtype=np.complex64)
        g = c.copy()
        oracle.cgemm("N", "N", m, n, 0, 1 + 0j, None, 3, None, 1, beta, g, ldc)
        view = g.reshape(n, ldc)
        if beta == 1:
            assert g.tobytes() == c.tobytes()
        elif beta == 0:
            assert np.all(view[:, :m] == 0)
        else:
            assert np.allclose(view[:, :m], beta * init_val)
        assert view[:, m:].tobytes() == c.reshape(n, ldc)[:, m:].tobytes()


# ---------------------------------------------------------------- rounding correction

def test_segment_cancellation_kat(oracle):
    """cgemm3m_test.cpp:212-240: +4096.1 x 660 then -4096.1 x 660 along K plus a
    residual at K=2047 must come back as the residual within 0.01 -- sequential
    FP32 accumulation does not (it drifts by ~0.015)."""
    size, tps = 2048, 33
    assert oracle.segment_span(size) == tps
    arow = np.zeros(size, np.complex64)
    bcol = np.zeros(size, np.complex64)
    arow[: 40 * tps] = 1
    bcol[: 20 * tps] = 4096.1
    bcol[20 * tps: 40 * tps] = -4096.1
    arow[size - 1] = 1
    for residual in (0.0, 1.0):
        bcol[size - 1] = residual
        got = oracle.recompute_dot(arow, bcol)
        assert abs(got.real - residual) <= 0.01
        assert abs(got.imag) <= 0.01
        seq = np.float32(0)
        for x, y in zip(arow.real, bcol.real):
            seq = np.float32(seq + np.float32(x * y))
        assert abs(float(seq) - residual) > 0.01  # why the correction exists


def test_selection_flags_the_kat_output(oracle):
    """The KAT's output C(0,0) is selected by the reference's screening formula
    (cgemm3m_rounding_kernel.cpp:43-100) from its partial-sum trajectory."""
    n, tps = 2048, 33
    terms = np.zeros(n, np.float64)
    terms[: 20 * tps] = 4096.1
    terms[20 * tps: 40 * tps] = -4096.1
    s = np.cumsum(terms)
    path = 0.0
    old = 0.0
    for k0 in range(0, n, 128):
        new = s[min(k0 + 128, n) - 1]
        path += 128 / 9 * (old * old + old * new + new * new)
        old = new
    e_row = float(40 * tps + 1)
    e_col = float(40 * tps) * 4096.1 ** 2
    var = 2.0 ** -48 * (path + e_row * e_col * oracle.bridge(n))
    assert 3.75 ** 2 * var >= 1e-4


def test_bridge_term(oracle):
    for n in (2048, 3000, 4096):
        expect = ((n // 128) * 128 * 128 + (n % 128) ** 2) / (18.0 * n * n)
        assert abs(oracle.bridge(n) - expect) <= 1e-6 * expect


def test_risk_select_recompute_small(oracle):
    """End-to-end restatement on a small square problem: energies, path,
    selection and recompute keep unflagged outputs and move flagged ones no
    further from FP64 than FP32 rounding allows."""
    n = 160
    rng = np.random.default_rng(5)
    a = (rng.standard_normal(n * n) * 300 + 1j * rng.standard_normal(n * n)).astype(np.complex64)
    b = (rng.standard_normal(n * n) * 300 + 1j * rng.standard_normal(n * n)).astype(np.complex64)
    path, c = oracle.risk_path(n, a, b)
    e = oracle.energy(n, "N", "N", a, n, b, n)
    A = oracle.unpack(a, n, n, n).astype(np.complex128)
    B = oracle.unpack(b, n, n, n).astype(np.complex128)
    assert np.allclose(e[:n], (np.abs(A) ** 2).sum(1), rtol=1e-5)
    assert np.allclose(e[n:], (np.abs(B) ** 2).sum(0), rtol=1e-5)
    flags, count = oracle.select(n, c, e, path)
    assert 0 < count <= n * n
    fixed = c.copy()
    oracle.recompute(n, "N", "N", a, n, b, n, flags, fixed)
    exact = (A @ B).T.reshape(-1)
    keep = flags == 0
    assert fixed[keep].tobytes() == c[keep].tobytes()
    err = np.abs(fixed - exact)
    assert err.max() <= 1e-3 * np.abs(exact).max()


# ---------------------------------------------------------------- case table

def test_case_table_integrity(cases):
    rows = cases["cases"]
    assert cases["count"] == 1200 == len(rows)
    names = [r["name"] for r in rows]
    assert len(set(names)) == len(names)
    assert sum(n.startswith("TC_PF_") for n in names) == 200
    pf = [r for r in rows if r["name"].startswith("TC_PF_")]
    assert all(r["alpha"] == [1.0, 0.0] and r["beta"] == [0.0, 0.0] for r in pf)
    assert sum(r["expect"] != "SUCCESS" for r in rows) == 16


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "T"), ("T", "C"), ("R", "N"), ("N", "C")])
def test_timing_build_gives_the_checkers_bytes(oracle, ta, tb):
    """The CPU-baseline build of the reference-order cgemm (no volatile stores,
    vectorised) computes the same bytes as the checker build."""
    m, n, k = 97, 61, 130
    al, be = complex(0.7, 0.3), complex(-1.0, 0.5)
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    a = oracle.make_matrix(ar, ac, ar + 3, "UNIFORM_1", 11)
    b = oracle.make_matrix(br, bc, br + 1, "UNIFORM_1", 12)
    c = oracle.make_matrix(m, n, m + 2, "UNIFORM_1", 13)
    c1, c2 = c.copy(), c.copy()
    oracle.cgemm(ta, tb, m, n, k, al, a, ar + 3, b, br + 1, be, c1, m + 2)
    oracle.cgemm_timing(ta, tb, m, n, k, al, a, ar + 3, b, br + 1, be, c2, m + 2)
    assert c1.tobytes() == c2.tobytes()
