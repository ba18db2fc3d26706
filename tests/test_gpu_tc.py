"""GPU parity of the tensor-core precision forms (3xTF32, split-BF16 x6/x9).

The tensor-core accumulation order inside an MMA is the hardware's, so these
forms are checked against FP64 rather than bit for bit (engine="packed" keeps
every call on the tensor cores; the planner may otherwise run a small problem
as plain FP32): the reference accuracy
criterion (cgemm3m_verify.h:22-84) against the FP64 result rounded to FP32, a
normwise-error bound, run-to-run bitwise determinism, and the precision forms'
promise -- normwise error vs FP64 no worse than the plain FP32 3M form on the
same inputs.
"""
import numpy as np
import pytest

from gpu_util import run, to_dev, to_host

pytestmark = pytest.mark.gpu

FORMS = ["tf32x3", "bf16x6", "bf16x9"]
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


def _check(oracle, out, c, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, ldc, bound):
    z = oracle.zgemm_numpy(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    golden = c.copy()
    golden.reshape(n, ldc)[:, :m] = z.T.astype(np.complex64)
    ok, re, im, pad = oracle.verify_cgemm3m(out, golden, c, m, n, ldc)
    assert ok, (re.__dict__, im.__dict__, pad)
    err = oracle.error_report(oracle.unpack(out, ldc, m, n), z)
    assert err["normwise"] < bound, err
    return err


@pytest.mark.parametrize("form", FORMS)
def test_tc_single_tile(cg3m, oracle, cuda, h, form):
    import torch

    m = n = 128
    k = 64
    a, lda, b, ldb, c, ldc = _operands(oracle, "N", "N", m, n, k, 0, "UNIFORM_1", 1)
    out, info = run(cg3m, h, torch, cuda, "N", "N", m, n, k, 1.0, a, lda, b, ldb, 0.0, c, ldc, form=form,
                    engine="packed")
    assert info["form"] == cg3m.FORM[form]
    _check(oracle, out, c, "N", "N", m, n, k, 1.0, a, lda, b, ldb, 0.0, ldc, 1e-6)
    assert h.device_status() == 0


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (130, 129, 70), (257, 300, 1000), (64, 200, 65)])
@pytest.mark.parametrize("ops", [("N", "N"), ("T", "C"), ("C", "T")])
def test_tc_edges(cg3m, oracle, cuda, h, form, shape, ops):
    import torch

    m, n, k = shape
    ta, tb = ops
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, ta, tb, m, n, k, 3, "UNIFORM_1", m + n + k)
    out, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form,
                 engine="packed")
    again, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form,
                   engine="packed")
    assert out.tobytes() == again.tobytes()
    _check(oracle, out, c, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, ldc, 2e-6)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("ta", OPS)
@pytest.mark.parametrize("tb", OPS)
def test_tc_nine_ops_padded(cg3m, oracle, cuda, h, form, ta, tb):
    import torch

    m, n, k = 1000, 777, 3001
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, ta, tb, m, n, k, 13, "UNIFORM_1", 9000 + 3 * OPS.index(ta) +
                                       OPS.index(tb))
    out, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form,
                 engine="packed")
    _check(oracle, out, c, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, ldc, 2e-6)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("parts", [2, 3, 4, 5])
def test_tc_forced_partitions(cg3m, oracle, cuda, h, form, parts):
    """CTA-pair kernel with a forced K split: 2..4 partitions merge inside the
    kernel through the tile's cluster (pack + GEMM), 5 through the merge kernel."""
    import torch

    m, n, k = 200, 150, 1500  # 24 blocks of 64: splits into 2, 3, 4 and 5 spans come out exact
    alpha, beta = complex(0.3, -1.25), complex(0.5, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, "T", "N", m, n, k, 2, "RANDOM_NORM_5_5", 77)
    out, info = run(cg3m, h, torch, cuda, "T", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form,
                    k_partitions=parts, engine="packed")
    assert info["k_partitions"] == parts and info["k_span"] % 64 == 0
    assert info["kernels"] == (2 if parts <= 4 else 3)
    again, _ = run(cg3m, h, torch, cuda, "T", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form,
                   k_partitions=parts, engine="packed")
    assert out.tobytes() == again.tobytes()
    _check(oracle, out, c, "T", "N", m, n, k, alpha, a, lda, b, ldb, beta, ldc, 2e-6)
    assert h.device_status() == 0


@pytest.mark.parametrize("form", FORMS)
def test_tc_long_k(cg3m, oracle, cuda, h, form):
    import torch

    m = n = 128
    k = 65536
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, "N", "N", m, n, k, 0, "UNIFORM_1", 4243)
    out, info = run(cg3m, h, torch, cuda, "N", "N", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form,
                    engine="packed")
    assert info["k_partitions"] > 1
    _check(oracle, out, c, "N", "N", m, n, k, alpha, a, lda, b, ldb, beta, ldc, 2e-6)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("size,rounding", [(1024, "off"), (2048, "off"), (3072, "off"), (4096, "off"),
                                           (2048, "auto"), (3072, "auto"), (4096, "auto")])
def test_tc_error_no_worse_than_plain(cg3m, oracle, cuda, h, form, size, rounding):
    """Precision-form data (Im scaled by 2^e, e in [-8, 8] per column, which
    stresses the cancellation in Im = P2-P0-P1), alpha=1, beta=0, NN -- the
    precision form's configuration at N = 2048, 3072, 4096: the tensor-core
    form's normwise error vs FP64 must not exceed the plain FP32 3M form's,
    with the rounding-correction pass off in both (only the products differ)
    and on in both (the drop-in's default gate admits these squares)."""
    import torch

    n = size
    A = to_dev(oracle.precision_matrix(n, n, 11), torch, cuda)
    B = to_dev(oracle.precision_matrix(n, n, 12), torch, cuda)
    C = torch.zeros(n * n, dtype=torch.complex64, device=cuda)
    ref = torch.empty(n * n, dtype=torch.complex128, device=cuda)
    h.zgemm_reference("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, ref)
    info = h.cgemm3m("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, form="fp32", rounding=rounding)
    assert info["rounding"] == (1 if rounding == "auto" else 0)
    plain = h.error_report(n, n, C, n, ref)
    h.cgemm3m("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, form=form, rounding=rounding, engine="packed")
    tc = h.error_report(n, n, C, n, ref)
    torch.cuda.synchronize()
    print(form, n, rounding, "plain", plain, "tc", tc)
    assert tc["normwise"] <= plain["normwise"], (plain, tc)
    assert tc["normwise"] < 1e-5
    del A, B, C, ref
    torch.cuda.empty_cache()


@pytest.mark.parametrize("form", FORMS)
def test_tc_small_problem_runs_plain_fp32(cg3m, oracle, cuda, h, form):
    """Planner's choice for a small tensor-core call: the one-launch FP32
    product (info reports form FP32, path 4), bit-identical to the FP32 form
    with the same K split, and within the reference criterion."""
    import torch

    m, n, k = 96, 80, 200
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    a, lda, b, ldb, c, ldc = _operands(oracle, "T", "C", m, n, k, 2, "UNIFORM_1", 616)
    out, info = run(cg3m, h, torch, cuda, "T", "C", m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, form=form)
    assert info["form"] == cg3m.FORM["fp32"] and info["path"] == 4
    model = c.copy()
    oracle.cgemm3m_fp32_model("T", "C", m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
    assert out.tobytes() == model.tobytes()
    _check(oracle, out, c, "T", "C", m, n, k, alpha, a, lda, b, ldb, beta, ldc, 2e-6)
