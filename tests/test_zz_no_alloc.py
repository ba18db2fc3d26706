"""cg3mCgemm3mNoAlloc, the entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc where they multiply -- code
running under a caching allocator that owns the device heap, or a hot loop
where an allocation would synchronize the device.  Its scratch is a fixed
device array inside the library instead of a workspace, so its result must be
exactly the drop-in's.  This file is collected last on purpose: if it fails,
a run that stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_no_alloc(cg3m, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    al, be = cg3m.cx(alpha), cg3m.cx(beta)
    return cg3m.lib.cg3mCgemm3mNoAlloc(ctypes.c_void_p(stream), cg3m.OP[ta], cg3m.OP[tb], m, n, k, ctypes.byref(al),
                                       cg3m.ptr(A), lda, cg3m.ptr(B), ldb, ctypes.byref(be), cg3m.ptr(C), ldc)


def test_no_alloc_matches_drop_in_twice(cg3m, oracle, cuda):
    import torch

    m, n, k = 300, 200, 257
    ta, tb = "T", "C"
    alpha, beta = complex(0.7, 0.3), complex(-1.0, 0.5)
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + 5, br + 3, m + 7
    a = oracle.make_matrix(ar, ac, lda, "UNIFORM_1", 31)
    b = oracle.make_matrix(br, bc, ldb, "UNIFORM_1", 32)
    c = oracle.make_matrix(m, n, ldc, "UNIFORM_1", 33)
    A = torch.from_numpy(a).to(cuda)
    B = torch.from_numpy(b).to(cuda)

    # the existing drop-in entry point
    h = cg3m.Handle(stream=torch.cuda.current_stream().cuda_stream)
    C_ref = torch.from_numpy(c.copy()).to(cuda)
    assert h.cgemm3m(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_ref, ldc, raw=True) == cg3m.SUCCESS
    torch.cuda.synchronize()
    expect = C_ref.cpu().numpy()

    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the second call starts from the first call's scratch contents
        C = torch.from_numpy(c.copy()).to(cuda)
        st = _call_no_alloc(cg3m, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
        torch.cuda.synchronize()
        assert st == cg3m.SUCCESS
        got = C.cpu().numpy()
        ok, re, im, pad = oracle.verify_cgemm3m(got, expect, c, m, n, ldc)
        assert ok, (re.__dict__, im.__dict__, pad)
        assert got.tobytes() == expect.tobytes()


# Shapes whose plan puts packed planes (and split partials) in the fixed array:
# config 1's 512^3 (K split merged in the GEMM's cluster), a fused square, a
# conjugated split, and a long-K split whose partials go through the merge
# kernel.
SCRATCH_CASES = [
    ("N", "N", 512, 512, 512, complex(1.5, -0.5), complex(0.25, 0.75)),
    ("N", "N", 1024, 1024, 1024, 1.0, 0.0),
    ("C", "N", 700, 600, 900, complex(0.7, 0.3), complex(-1.0, 0.5)),
    ("N", "T", 64, 64, 16384, complex(0.5, 0.5), 0.0),
]


@pytest.mark.parametrize("ta,tb,m,n,k,alpha,beta", SCRATCH_CASES)
def test_no_alloc_uses_its_scratch_and_matches_drop_in(cg3m, oracle, cuda, ta, tb, m, n, k, alpha, beta):
    """The planner puts this call's packed planes (and any partials) in the
    fixed array; two calls in a row give the drop-in's bytes."""
    import torch

    plan = cg3m.plan(ta, tb, m, n, k, alpha, beta)
    assert plan["path"] in (2, 3) and 0 < plan["workspace_bytes"] <= (32 << 20) - 256
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar, br, m + 3
    a = oracle.make_matrix(ar, ac, lda, "UNIFORM_1", 41)
    b = oracle.make_matrix(br, bc, ldb, "UNIFORM_1", 42)
    c = oracle.make_matrix(m, n, ldc, "UNIFORM_1", 43)
    A = torch.from_numpy(a).to(cuda)
    B = torch.from_numpy(b).to(cuda)
    h = cg3m.Handle(stream=torch.cuda.current_stream().cuda_stream)
    C_ref = torch.from_numpy(c.copy()).to(cuda)
    assert h.cgemm3m(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_ref, ldc, raw=True) == cg3m.SUCCESS
    torch.cuda.synchronize()
    expect = C_ref.cpu().numpy()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        C = torch.from_numpy(c.copy()).to(cuda)
        st = _call_no_alloc(cg3m, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
        torch.cuda.synchronize()
        assert st == cg3m.SUCCESS
        assert C.cpu().numpy().tobytes() == expect.tobytes()
    flags = ctypes.c_int(-1)
    assert cg3m.lib.cg3mGetDeviceStatus(None, ctypes.byref(flags)) == cg3m.SUCCESS
    assert flags.value == 0


def test_no_alloc_status_word_reports_a_wait_that_gave_up(cg3m, oracle, cuda):
    """A bounded wait that runs out sets the allocation-free entry point's
    status word; cg3mGetDeviceStatus(NULL) reports it once and clears it, and
    the next call is unaffected."""
    import torch

    gave_up = ctypes.c_int(0)
    assert cg3m.lib.cg3mDiagBoundedWait(None, 1_000_000, ctypes.byref(gave_up)) == cg3m.SUCCESS
    assert gave_up.value == 1
    flags = ctypes.c_int(0)
    assert cg3m.lib.cg3mGetDeviceStatus(None, ctypes.byref(flags)) == cg3m.SUCCESS
    assert flags.value == 1
    assert cg3m.lib.cg3mGetDeviceStatus(None, ctypes.byref(flags)) == cg3m.SUCCESS
    assert flags.value == 0
    m = n = k = 512
    a = oracle.make_matrix(m, k, m, "UNIFORM_1", 51)
    b = oracle.make_matrix(k, n, k, "UNIFORM_1", 52)
    A, B = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    C = torch.zeros(m * n, dtype=torch.complex64, device=cuda)
    st = _call_no_alloc(cg3m, torch.cuda.current_stream().cuda_stream, "N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m)
    torch.cuda.synchronize()
    assert st == cg3m.SUCCESS
    model = np.zeros(m * n, np.complex64)
    oracle.cgemm3m_fp32_model("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, model, m,
                              span=cg3m.plan("N", "N", m, n, k)["k_span"])
    assert C.cpu().numpy().tobytes() == model.tobytes()
    assert cg3m.lib.cg3mGetDeviceStatus(None, ctypes.byref(flags)) == cg3m.SUCCESS
    assert flags.value == 0


def test_no_alloc_rejects_oversized_problem(cg3m, cuda):
    import torch

    m = n = k = 2048  # packed planes alone need 96 MiB, more than the fixed array
    A = torch.zeros(m * k, dtype=torch.complex64, device=cuda)
    B = torch.zeros(k * n, dtype=torch.complex64, device=cuda)
    C = torch.full((m * n,), complex(1.0, 2.0), dtype=torch.complex64, device=cuda)
    st = _call_no_alloc(cg3m, torch.cuda.current_stream().cuda_stream, "N", "N", m, n, k, 1.0, A, m, B, k,
                        0.5, C, m)
    torch.cuda.synchronize()
    assert st == cg3m.INVALID_VALUE
    assert bool(torch.all(C == complex(1.0, 2.0)))
