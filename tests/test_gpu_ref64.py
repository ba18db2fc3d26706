"""The device FP64 yardstick, pinned to numpy.

cg3mZgemmReference (the FP64 product every error figure is measured against)
and cg3mErrorReport (the normwise / componentwise report) run on the GPU;
here both are checked against numpy complex128 (oracle.zgemm_numpy and
oracle.error_report): all nine op pairs with padded leading dimensions and
general alpha/beta at 512^3, and the precision-form data at 2048^3.  The
tolerance is FP64-level: the products differ only in summation order.
"""
import numpy as np
import pytest

from gpu_util import to_dev

pytestmark = pytest.mark.gpu

OPS = [(a, b) for a in "NTC" for b in "NTC"]


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _fp64_gap(x, z):
    """(normwise, worst element relative to the largest) distance of two FP64 results."""
    d = np.abs(x - z)
    return float(np.linalg.norm(x - z) / np.linalg.norm(z)), float(d.max() / np.abs(z).max())


@pytest.mark.parametrize("ta,tb", OPS)
def test_zgemm_reference_matches_numpy(cg3m, oracle, cuda, h, ta, tb):
    import torch

    m = n = k = 512
    # the API takes alpha and beta as FP32: the exact product is with those values
    alpha = complex(np.float32(0.7), np.float32(0.3))
    beta = complex(np.float32(-1.0), np.float32(0.5))
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + 13, br + 13, m + 13
    a = oracle.make_matrix(ar, ac, lda, "UNIFORM_1", 101)
    b = oracle.make_matrix(br, bc, ldb, "UNIFORM_1", 102)
    c = oracle.make_matrix(m, n, ldc, "UNIFORM_1", 103)
    out = torch.empty(m * n, dtype=torch.complex128, device=cuda)
    h.zgemm_reference(ta, tb, m, n, k, alpha, to_dev(a, torch, cuda), lda, to_dev(b, torch, cuda), ldb, beta,
                      to_dev(c, torch, cuda), ldc, out)
    torch.cuda.synchronize()
    x = out.cpu().numpy().reshape(n, m).T
    z = oracle.zgemm_numpy(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    normwise, worst = _fp64_gap(x, z)
    assert normwise <= 1e-13 and worst <= 1e-13, (normwise, worst)


def test_zgemm_reference_and_error_report_on_precision_data(cg3m, oracle, cuda, h):
    """2048^3 precision-form data (Im scaled by 2^e per column): the device
    FP64 product against numpy, and the device error report of an FP32 result
    against the same report computed on the host, entry by entry."""
    import torch

    n = 2048
    a = oracle.precision_matrix(n, n, 11)
    b = oracle.precision_matrix(n, n, 12)
    A, B = to_dev(a, torch, cuda), to_dev(b, torch, cuda)
    C = torch.zeros(n * n, dtype=torch.complex64, device=cuda)
    ref = torch.empty(n * n, dtype=torch.complex128, device=cuda)
    h.zgemm_reference("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, ref)
    h.cgemm3m("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, form="fp32", rounding="off")
    rep = h.error_report(n, n, C, n, ref)
    torch.cuda.synchronize()
    x = ref.cpu().numpy().reshape(n, n).T
    z = oracle.zgemm_numpy("N", "N", n, n, n, 1.0, a, n, b, n, 0.0, np.zeros(n * n, np.complex64), n)
    normwise, worst = _fp64_gap(x, z)
    assert normwise <= 1e-13 and worst <= 1e-13, (normwise, worst)
    got = oracle.unpack(C.cpu().numpy(), n, n, n)
    host = oracle.error_report(got, x)
    for key in ("normwise", "comp_re", "comp_im", "abs_re", "abs_im"):
        assert rep[key] == pytest.approx(host[key], rel=1e-9, abs=0.0), (key, rep[key], host[key])
    # and against numpy's own FP64 product: the same figures to FP64 precision
    host_np = oracle.error_report(got, z)
    assert rep["normwise"] == pytest.approx(host_np["normwise"], rel=1e-6)
