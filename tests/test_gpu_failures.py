"""Failure handling without faulting the GPU.

The reference maps platform failures to statuses (cgemm_host.cpp:109-127:
workspace allocation -> ALLOC_FAILED) and its test gate kills hung processes
by timeout (test_gate.py:72-87).  Here the failures are made on purpose in
the accepted forms: a device allocation the library is told to fail (host
side), and a bounded wait that cannot complete (an mbarrier nothing arrives
on, with a 1 ms limit), which must give up, set the status word and return.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _operands(oracle, torch, cuda, m, n, k, seed):
    a = oracle.make_matrix(m, k, m, "UNIFORM_1", seed)
    b = oracle.make_matrix(k, n, k, "UNIFORM_1", seed + 1)
    return a, b, torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)


def test_workspace_allocation_failure_is_reported_and_recovers(cg3m, oracle, cuda):
    """Workspace growth that fails returns ALLOC_FAILED with C untouched; the
    next call (allocation allowed again) computes the exact result."""
    import torch

    m = n = k = 2048  # needs far more than the 32 MiB default workspace
    a, b, A, B = _operands(oracle, torch, cuda, m, n, k, 61)
    stream = torch.cuda.current_stream().cuda_stream
    h = cg3m.Handle(stream=stream)
    small = torch.zeros(64 * 64, dtype=torch.complex64, device=cuda)
    assert h.cgemm3m("N", "N", 64, 64, 64, 1.0, A, m, B, k, 0.0, small, 64, raw=True) == cg3m.SUCCESS
    torch.cuda.synchronize()
    sentinel = complex(3.0, -7.0)
    C = torch.full((m * n,), sentinel, dtype=torch.complex64, device=cuda)
    assert cg3m.lib.cg3mDiagFailAllocations(1) == cg3m.SUCCESS
    try:
        st = h.cgemm3m("N", "N", m, n, k, complex(1.5, -0.5), A, m, B, k, complex(0.25, 0.75), C, m, raw=True)
    finally:
        cg3m.lib.cg3mDiagFailAllocations(0)
    torch.cuda.synchronize()
    assert st == cg3m.ALLOC_FAILED
    assert bool(torch.all(C == sentinel))
    st = h.cgemm3m("N", "N", m, n, k, complex(1.5, -0.5), A, m, B, k, complex(0.25, 0.75), C, m, raw=True)
    torch.cuda.synchronize()
    assert st == cg3m.SUCCESS
    info = cg3m.plan("N", "N", m, n, k, complex(1.5, -0.5), complex(0.25, 0.75))
    model = np.full(m * n, sentinel, np.complex64)
    oracle.cgemm3m_fp32_model("N", "N", m, n, k, complex(1.5, -0.5), a, m, b, k, complex(0.25, 0.75), model, m,
                              span=info["k_span"])
    assert C.cpu().numpy().tobytes() == model.tobytes()
    assert h.device_status() == 0


def test_first_binding_allocation_failure(cg3m, cuda):
    """A fresh handle whose first device allocation fails reports ALLOC_FAILED
    and binds on a later call."""
    import torch

    h = cg3m.Handle(stream=torch.cuda.current_stream().cuda_stream)
    C = torch.ones(16 * 16, dtype=torch.complex64, device=cuda)
    assert cg3m.lib.cg3mDiagFailAllocations(1) == cg3m.SUCCESS
    try:
        # k == 0: a beta-scale only call, which still binds the handle first
        st = h.cgemm3m("N", "N", 16, 16, 0, 1.0, None, 16, None, 1, 2.0, C, 16, raw=True)
    finally:
        cg3m.lib.cg3mDiagFailAllocations(0)
    assert st == cg3m.ALLOC_FAILED
    torch.cuda.synchronize()
    assert bool(torch.all(C == 1.0))
    st = h.cgemm3m("N", "N", 16, 16, 0, 1.0, None, 16, None, 1, 2.0, C, 16, raw=True)
    torch.cuda.synchronize()
    assert st == cg3m.SUCCESS
    assert bool(torch.all(C == 2.0))


def test_bounded_wait_gives_up_sets_status_and_context_survives(cg3m, oracle, cuda):
    """The wait every pipeline kernel uses gives up after its limit on a
    barrier nothing arrives on: the kernel returns, bit 1 of the handle's
    status word is set (read once, then clear), and a following tensor-core
    call on the same handle is correct."""
    import torch

    h = cg3m.Handle(stream=torch.cuda.current_stream().cuda_stream)
    gave_up = ctypes.c_int(0)
    assert cg3m.lib.cg3mDiagBoundedWait(h.h, 1_000_000, ctypes.byref(gave_up)) == cg3m.SUCCESS
    assert gave_up.value == 1
    assert h.device_status() == 1
    assert h.device_status() == 0
    m = n = k = 256
    a, b, A, B = _operands(oracle, torch, cuda, m, n, k, 71)
    C = torch.zeros(m * n, dtype=torch.complex64, device=cuda)
    h.cgemm3m("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, form="bf16x6", rounding="off", engine="packed")
    torch.cuda.synchronize()
    z = oracle.zgemm_numpy("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, np.zeros(m * n, np.complex64), m)
    err = oracle.error_report(oracle.unpack(C.cpu().numpy(), m, m, n), z)
    assert err["normwise"] < 1e-6
    assert h.device_status() == 0


def test_bounded_wait_limit_is_validated(cg3m, cuda):
    gave_up = ctypes.c_int(0)
    assert cg3m.lib.cg3mDiagBoundedWait(None, 0, ctypes.byref(gave_up)) == cg3m.INVALID_VALUE
    assert cg3m.lib.cg3mDiagBoundedWait(None, 20_000_000_000, ctypes.byref(gave_up)) == cg3m.INVALID_VALUE
