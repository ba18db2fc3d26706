"""GPU parity of the on-chip product family: cg3mCgemm3mStridedBatched and
cg3mCgemm (the reference's aclblasCgemm3mStridedBatched and aclblasCgemm).

Bars:
  * bit-exact against the oracle's model of the family
    (oracle_cgemm_modes_fp32: 3M or four products, K partitions of the plan,
    non-finite repair) on ragged, padded, all-op problems;
  * the reference's strided semantics (blas/gemm/README.md:809-907): zero and
    negative strides, overlapping outputs updated in batch order, the
    identity example (A = I gives C = B bitwise), bitwise repeatability;
  * the non-finite repair: 3M products that overflow in the sums Ar+Ai, Br+Bi
    come out as the finite four-product value;
  * cgemm against the reference-order FP32 cgemm with the reference criterion.
"""
import numpy as np
import pytest

from gpu_util import same_bits, to_dev, to_host

pytestmark = pytest.mark.gpu

OPS = ["N", "T", "C"]


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _strided_buffers(oracle, ta, tb, m, n, k, batch, pad, fill, seed):
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + pad, br + pad, m + pad
    sA, sB, sC = lda * ac + 3, ldb * bc + 5, ldc * n + 7
    # batches laid out at the strides, with gaps between them
    A = np.zeros(sA * batch, np.complex64)
    B = np.zeros(sB * batch, np.complex64)
    C = np.zeros(sC * batch, np.complex64)
    for i in range(batch):
        A[i * sA:i * sA + lda * ac] = oracle.make_matrix(ar, ac, lda, fill, seed + 10 * i)
        B[i * sB:i * sB + ldb * bc] = oracle.make_matrix(br, bc, ldb, fill, seed + 10 * i + 1)
        C[i * sC:i * sC + ldc * n] = oracle.make_matrix(m, n, ldc, fill, seed + 10 * i + 2)
    return A, lda, sA, B, ldb, sB, C, ldc, sC


@pytest.mark.parametrize("ta", OPS)
@pytest.mark.parametrize("tb", OPS)
def test_strided_bit_exact_vs_model(cg3m, oracle, cuda, h, ta, tb):
    import torch

    m, n, k, batch = 70, 45, 300, 5
    alpha, beta = complex(0.7, 0.3), complex(-1, 0.5)
    A, lda, sA, B, ldb, sB, C, ldc, sC = _strided_buffers(oracle, ta, tb, m, n, k, batch, 3, "UNIFORM_1", 100)
    dC = to_dev(C, torch, cuda)
    st = h.cgemm3m_strided_batched(ta, tb, m, n, k, alpha, to_dev(A, torch, cuda), lda, sA, to_dev(B, torch, cuda),
                                   ldb, sB, beta, dC, ldc, sC, batch)
    assert st == cg3m.SUCCESS
    torch.cuda.synchronize()
    out = to_host(dC)
    plan = cg3m.plan_onchip(m, n, k, 0, batch, torch.cuda.get_device_properties(cuda).multi_processor_count)
    want = C.copy()
    for i in range(batch):
        ci = want[i * sC:i * sC + ldc * n].copy()
        oracle.cgemm_modes_model(0, 1, ta, tb, m, n, k, alpha, A[i * sA:], lda, B[i * sB:], ldb, beta, ci, ldc,
                                 span=plan["k_span"] if plan["k_partitions"] > 1 else 0)
        want[i * sC:i * sC + ldc * n] = ci
    assert same_bits(out, want)
    # repeatable bit for bit
    dC2 = to_dev(C, torch, cuda)
    h.cgemm3m_strided_batched(ta, tb, m, n, k, alpha, to_dev(A, torch, cuda), lda, sA, to_dev(B, torch, cuda), ldb,
                              sB, beta, dC2, ldc, sC, batch)
    torch.cuda.synchronize()
    assert to_host(dC2).tobytes() == out.tobytes()


def test_strided_long_k_split_and_model(cg3m, oracle, cuda, h):
    import torch

    m, n, k, batch = 64, 64, 4096, 2
    A, lda, sA, B, ldb, sB, C, ldc, sC = _strided_buffers(oracle, "N", "C", m, n, k, batch, 0, "RANDOM_NORM_5_5", 7)
    plan = cg3m.plan_onchip(m, n, k, 0, batch, torch.cuda.get_device_properties(cuda).multi_processor_count)
    assert plan["k_partitions"] > 1
    dC = to_dev(C, torch, cuda)
    assert h.cgemm3m_strided_batched("N", "C", m, n, k, 1.0, to_dev(A, torch, cuda), lda, sA, to_dev(B, torch, cuda),
                                     ldb, sB, 0.0, dC, ldc, sC, batch) == cg3m.SUCCESS
    torch.cuda.synchronize()
    out = to_host(dC)
    want = C.copy()
    for i in range(batch):
        ci = want[i * sC:i * sC + ldc * n].copy()
        oracle.cgemm_modes_model(0, 1, "N", "C", m, n, k, 1.0, A[i * sA:], lda, B[i * sB:], ldb, 0.0, ci, ldc,
                                 span=plan["k_span"])
        want[i * sC:i * sC + ldc * n] = ci
    assert same_bits(out, want)


def test_strided_identity_example(cg3m, cuda, h):
    """blas/gemm/README.md:854-907: two 2x2 batches, A = I, C must equal B bitwise."""
    import torch

    a = np.array([1, 0, 0, 1, 1, 0, 0, 1], np.complex64)
    b = np.array([1, 2, 3, 4, 5, 6, 7, 8], np.complex64)
    dC = torch.zeros(8, dtype=torch.complex64, device=cuda)
    assert h.cgemm3m_strided_batched("N", "N", 2, 2, 2, 1.0, to_dev(a, torch, cuda), 2, 4, to_dev(b, torch, cuda), 2,
                                     4, 0.0, dC, 2, 4, 2) == cg3m.SUCCESS
    torch.cuda.synchronize()
    assert to_host(dC).tobytes() == b.tobytes()


def test_strided_overlap_in_batch_order(cg3m, oracle, cuda, h):
    """strideC = 0: every batch updates the same C in batch order."""
    import torch

    m, n, k, batch = 33, 17, 40, 4
    alpha, beta = complex(0.5, -0.25), complex(0.75, 0.5)
    a = np.concatenate([oracle.make_matrix(m, k, m, "UNIFORM_1", 40 + i) for i in range(batch)])
    b = np.concatenate([oracle.make_matrix(k, n, k, "UNIFORM_1", 50 + i) for i in range(batch)])
    c = oracle.make_matrix(m, n, m, "UNIFORM_1", 60)
    dC = to_dev(c, torch, cuda)
    assert h.cgemm3m_strided_batched("N", "N", m, n, k, alpha, to_dev(a, torch, cuda), m, m * k,
                                     to_dev(b, torch, cuda), k, k * n, beta, dC, m, 0, batch) == cg3m.SUCCESS
    torch.cuda.synchronize()
    # overlapping outputs run one batch per launch: the one-problem plan
    plan = cg3m.plan_onchip(m, n, k, 0, 1, torch.cuda.get_device_properties(cuda).multi_processor_count)
    span = plan["k_span"] if plan["k_partitions"] > 1 else 0
    want = c.copy()
    for i in range(batch):
        oracle.cgemm_modes_model(0, 1, "N", "N", m, n, k, alpha, a[i * m * k:], m, b[i * k * n:], k, beta, want, m,
                                 span=span)
    assert same_bits(to_host(dC), want)


def test_strided_negative_and_zero_strides(cg3m, oracle, cuda, h):
    """A shared by every batch (strideA = 0), B walked backwards (strideB < 0)."""
    import torch

    m, n, k, batch = 20, 30, 50, 3
    a = oracle.make_matrix(m, k, m, "UNIFORM_1", 70)
    b = np.concatenate([oracle.make_matrix(k, n, k, "UNIFORM_1", 80 + i) for i in range(batch)])
    c = np.zeros(m * n * batch, np.complex64)
    dB = to_dev(b, torch, cuda)
    dC = to_dev(c, torch, cuda)
    last = dB[(batch - 1) * k * n:]  # B_0 is the last block, B_i = B_0 - i*k*n
    assert h.cgemm3m_strided_batched("N", "N", m, n, k, 1.0, to_dev(a, torch, cuda), m, 0, last, k, -k * n, 0.0, dC,
                                     m, m * n, batch) == cg3m.SUCCESS
    torch.cuda.synchronize()
    out = to_host(dC)
    for i in range(batch):
        want = np.zeros(m * n, np.complex64)
        bi = b[(batch - 1 - i) * k * n:]
        oracle.cgemm_modes_model(0, 1, "N", "N", m, n, k, 1.0, a, m, bi, k, 0.0, want, m)
        assert same_bits(out[i * m * n:(i + 1) * m * n], want), i


def test_nonfinite_repair(cg3m, oracle, cuda, h):
    """Entries near the FP32 maximum make Ar+Ai overflow: the 3M product is
    non-finite, the repaired output equals the finite four-product sum."""
    import torch

    m, n, k = 40, 24, 64
    rng = np.random.default_rng(5)
    a = (rng.uniform(-1, 1, m * k) + 1j * rng.uniform(-1, 1, m * k)).astype(np.complex64)
    b = (rng.uniform(-1, 1, k * n) + 1j * rng.uniform(-1, 1, k * n)).astype(np.complex64)
    hot = rng.choice(m * k, 12, replace=False)
    a[hot] = np.complex64(complex(2.5e38, 2.5e38))
    b *= np.float32(1e-6)
    c = np.zeros(m * n, np.complex64)
    dC = to_dev(c, torch, cuda)
    assert h.cgemm3m_strided_batched("N", "N", m, n, k, 1.0, to_dev(a, torch, cuda), m, 0, to_dev(b, torch, cuda), k,
                                     0, 0.0, dC, m, 0, 1) == cg3m.SUCCESS
    torch.cuda.synchronize()
    out = to_host(dC)
    plan = cg3m.plan_onchip(m, n, k, 0, 1, torch.cuda.get_device_properties(cuda).multi_processor_count)
    span = plan["k_span"] if plan["k_partitions"] > 1 else 0
    want = c.copy()
    oracle.cgemm_modes_model(0, 1, "N", "N", m, n, k, 1.0, a, m, b, k, 0.0, want, m, span=span)
    assert same_bits(out, want)
    plain = c.copy()
    oracle.cgemm_modes_model(0, 0, "N", "N", m, n, k, 1.0, a, m, b, k, 0.0, plain, m, span=span)
    assert not np.all(np.isfinite(plain.view(np.float32)))  # 3M alone overflows ...
    assert np.all(np.isfinite(out.view(np.float32)))        # ... the repaired output does not


@pytest.mark.parametrize("fill", ["VALUE_NORM_INF", "VALUE_NORM_NAN", "RANDOM_EXTREME"])
def test_strided_nonfinite_fills_match_model(cg3m, oracle, cuda, h, fill):
    import torch

    m = n = k = 32
    A, lda, sA, B, ldb, sB, C, ldc, sC = _strided_buffers(oracle, "N", "N", m, n, k, 2, 0, fill, 300)
    dC = to_dev(C, torch, cuda)
    assert h.cgemm3m_strided_batched("N", "N", m, n, k, 1.0, to_dev(A, torch, cuda), lda, sA, to_dev(B, torch, cuda),
                                     ldb, sB, complex(0, 1), dC, ldc, sC, 2) == cg3m.SUCCESS
    torch.cuda.synchronize()
    want = C.copy()
    for i in range(2):
        ci = want[i * sC:i * sC + ldc * n].copy()
        oracle.cgemm_modes_model(0, 1, "N", "N", m, n, k, 1.0, A[i * sA:], lda, B[i * sB:], ldb, complex(0, 1), ci,
                                 ldc)
        want[i * sC:i * sC + ldc * n] = ci
    assert same_bits(to_host(dC), want)


CGEMM_CASES = [
    ("N", "N", 512, 512, 512, complex(1.5, -0.5), complex(0.25, 0.75), 0),
    ("T", "C", 100, 77, 301, complex(0.7, 0.3), complex(-1, 0.5), 13),
    ("C", "T", 64, 200, 1000, complex(1, 0), complex(0, 0), 2),  # unit: three products + repair
    ("N", "T", 129, 33, 17, complex(0, 1), complex(1, 0), 1),
]


@pytest.mark.parametrize("case", CGEMM_CASES, ids=[f"{c[0]}{c[1]}-{c[2]}x{c[3]}x{c[4]}" for c in CGEMM_CASES])
def test_cgemm_bit_exact_and_reference_criterion(cg3m, oracle, cuda, h, case):
    import torch

    ta, tb, m, n, k, alpha, beta, pad = case
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + pad, br + pad, m + pad
    a = oracle.make_matrix(ar, ac, lda, "RANDOM_NORM_5_5", 1)
    b = oracle.make_matrix(br, bc, ldb, "RANDOM_NORM_5_5", 2)
    c = oracle.make_matrix(m, n, ldc, "RANDOM_NORM_5_5", 3)
    dC = to_dev(c, torch, cuda)
    assert h.cgemm(ta, tb, m, n, k, alpha, to_dev(a, torch, cuda), lda, to_dev(b, torch, cuda), ldb, beta, dC,
                   ldc) == cg3m.SUCCESS
    torch.cuda.synchronize()
    out = to_host(dC)
    unit = alpha == 1 and beta == 0
    mode = 0 if unit else 1
    # unit: three products + repair on the FP32 planner's engine (plan mode 2)
    plan = cg3m.plan_onchip(m, n, k, 2 if unit else 1, 1, torch.cuda.get_device_properties(cuda).multi_processor_count)
    want = c.copy()
    oracle.cgemm_modes_model(mode, 1 if unit else 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, want, ldc,
                             span=plan["k_span"] if plan["k_partitions"] > 1 else 0)
    assert same_bits(out, want)
    golden = c.copy()
    oracle.cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, golden, ldc)
    ok, re, im, padok = oracle.verify_cgemm3m(out, golden, c, m, n, ldc)
    assert ok, (re.__dict__, im.__dict__, padok)


def _table_rows(cases, limit=3_000_000):
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


def test_cgemm_case_table_rows(cg3m, oracle, cuda, h, cases):
    """The reference's case table through cg3mCgemm (its legacy aclblasCgemm
    regression): reference criterion vs reference-order cgemm, padding bytes,
    determinism, and bit-exactness vs the family's model."""
    import torch

    rows = _table_rows(cases)
    assert len(rows) > 500
    sms = torch.cuda.get_device_properties(cuda).multi_processor_count
    failures = []
    for cs in rows:
        ta, tb, m, n, k = cs["transa"], cs["transb"], cs["m"], cs["n"], cs["k"]
        ar, ac = oracle.stored_shape(ta, m, k)
        br, bc = oracle.stored_shape(tb, k, n)
        a = oracle.make_matrix(ar, ac, cs["lda"], cs["a_fill"], cs["seed"])
        b = oracle.make_matrix(br, bc, cs["ldb"], cs["b_fill"], cs["seed"] + 1)
        c = oracle.make_matrix(m, n, cs["ldc"], cs["c_fill"], cs["seed"] + 2)
        alpha, beta = complex(*cs["alpha"]), complex(*cs["beta"])
        outs = []
        for _ in range(2):
            dC = to_dev(c, torch, cuda)
            st = h.cgemm(ta, tb, m, n, k, alpha, to_dev(a, torch, cuda), cs["lda"],
                         to_dev(b, torch, cuda), cs["ldb"], beta, dC, cs["ldc"])
            torch.cuda.synchronize()
            if st != cg3m.SUCCESS:
                failures.append((cs["name"], "status", st))
                break
            outs.append(to_host(dC))
        if len(outs) < 2:
            continue
        out = outs[0]
        golden = c.copy()
        oracle.cgemm(ta, tb, m, n, k, alpha, a, cs["lda"], b, cs["ldb"], beta, golden, cs["ldc"])
        ok, re, im, pad = oracle.verify_cgemm3m(out, golden, c, m, n, cs["ldc"])
        if not ok:
            failures.append((cs["name"], "criterion", re.__dict__, im.__dict__, pad))
        if not same_bits(out, outs[1]):
            failures.append((cs["name"], "nondeterministic"))
        if m and n and k and alpha != 0:
            unit = alpha == 1 and beta == 0
            mode = 0 if unit else 1
            plan = cg3m.plan_onchip(m, n, k, 2 if unit else 1, 1, sms)
            model = c.copy()
            oracle.cgemm_modes_model(mode, 1 if unit else 0, ta, tb, m, n, k, alpha, a, cs["lda"], b, cs["ldb"], beta,
                                     model, cs["ldc"], span=plan["k_span"] if plan["k_partitions"] > 1 else 0)
            if not same_bits(out, model):
                failures.append((cs["name"], "model"))
    assert not failures, failures[:10]


def test_strided_case_table_rows(cg3m, oracle, cuda, h, cases):
    """Every 4th successful case-table row as a strided batch of two (second
    batch with its own data): reference criterion per batch and bits of the
    family's model."""
    import torch

    rows = _table_rows(cases, limit=1_000_000)[::4]
    sms = torch.cuda.get_device_properties(cuda).multi_processor_count
    failures = []
    for cs in rows:
        ta, tb, m, n, k = cs["transa"], cs["transb"], cs["m"], cs["n"], cs["k"]
        ar, ac = oracle.stored_shape(ta, m, k)
        br, bc = oracle.stored_shape(tb, k, n)
        lda, ldb, ldc = cs["lda"], cs["ldb"], cs["ldc"]
        sA, sB, sC = lda * ac, ldb * bc, ldc * n
        a = np.concatenate([oracle.make_matrix(ar, ac, lda, cs["a_fill"], cs["seed"] + 10 * t) for t in range(2)])
        b = np.concatenate([oracle.make_matrix(br, bc, ldb, cs["b_fill"], cs["seed"] + 10 * t + 1) for t in range(2)])
        c = np.concatenate([oracle.make_matrix(m, n, ldc, cs["c_fill"], cs["seed"] + 10 * t + 2) for t in range(2)])
        alpha, beta = complex(*cs["alpha"]), complex(*cs["beta"])
        dC = to_dev(c, torch, cuda)
        st = h.cgemm3m_strided_batched(ta, tb, m, n, k, alpha, to_dev(a, torch, cuda), lda, sA,
                                       to_dev(b, torch, cuda), ldb, sB, beta, dC, ldc, sC, 2)
        torch.cuda.synchronize()
        if st != cg3m.SUCCESS:
            failures.append((cs["name"], "status", st))
            continue
        out = to_host(dC)
        plan = cg3m.plan_onchip(m, n, k, 0, 2, sms) if m and n and k else None
        for t in range(2):
            ct = c[t * sC:(t + 1) * sC]
            ot = out[t * sC:(t + 1) * sC]
            golden = ct.copy()
            oracle.cgemm(ta, tb, m, n, k, alpha, a[t * sA:], lda, b[t * sB:], ldb, beta, golden, ldc)
            ok, re, im, pad = oracle.verify_cgemm3m(ot, golden, ct, m, n, ldc)
            if not ok:
                failures.append((cs["name"], t, "criterion", re.__dict__, im.__dict__, pad))
            if m and n and k and alpha != 0:
                model = ct.copy()
                oracle.cgemm_modes_model(0, 1, ta, tb, m, n, k, alpha, a[t * sA:], lda, b[t * sB:], ldb, beta, model,
                                         ldc, span=plan["k_span"] if plan["k_partitions"] > 1 else 0)
                if not same_bits(ot, model):
                    failures.append((cs["name"], t, "model"))
    assert not failures, failures[:10]


def test_cgemm_unit_packed_engine_repair_pass(cg3m, oracle, cuda, h):
    """cg3mCgemm with alpha = 1, beta = 0 on a shape the planner gives to the
    packed engine: entries near the FP32 maximum make some three-product sums
    overflow, and the GEMM's epilogue recomputes exactly those outputs with the
    four-product sum before storing them -- the same bits as the on-chip
    family's model."""
    import torch

    m, n, k = 600, 400, 500
    plan = cg3m.plan_onchip(m, n, k, 2, 1, torch.cuda.get_device_properties(cuda).multi_processor_count)
    assert plan["path"] in (2, 3) and plan["kernels"] == (2 if plan["path"] == 2 else 2 + (plan["k_partitions"] > 8))
    rng = np.random.default_rng(17)
    a = (rng.uniform(-1, 1, m * k) + 1j * rng.uniform(-1, 1, m * k)).astype(np.complex64)
    b = (rng.uniform(-1, 1, k * n) + 1j * rng.uniform(-1, 1, k * n)).astype(np.complex64)
    hot = rng.choice(m * k, 40, replace=False)
    a[hot] = np.complex64(complex(2.5e38, 2.5e38))
    b *= np.float32(1e-6)
    c = np.zeros(m * n, np.complex64)
    dC = to_dev(c, torch, cuda)
    assert h.cgemm("N", "N", m, n, k, 1.0, to_dev(a, torch, cuda), m, to_dev(b, torch, cuda), k, 0.0, dC,
                   m) == cg3m.SUCCESS
    torch.cuda.synchronize()
    out = to_host(dC)
    span = plan["k_span"] if plan["k_partitions"] > 1 else 0
    want = c.copy()
    oracle.cgemm_modes_model(0, 1, "N", "N", m, n, k, 1.0, a, m, b, k, 0.0, want, m, span=span)
    assert same_bits(out, want)
    plain = c.copy()
    oracle.cgemm_modes_model(0, 0, "N", "N", m, n, k, 1.0, a, m, b, k, 0.0, plain, m, span=span)
    assert not np.all(np.isfinite(plain.view(np.float32)))  # the three-product sums overflow ...
    assert np.all(np.isfinite(out.view(np.float32)))        # ... the repaired outputs do not
