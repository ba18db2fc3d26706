"""GPU parity of the host-buffer entry point (cg3mCgemm3mHost).

Its result must be the bytes the device call (cg3mCgemm3mEx on device copies)
gives for the whole problem, whatever the panel count: the panels keep the
whole problem's K split, and the rounding-correction case runs as one panel.
C rows past m on the host stay untouched.
"""
import numpy as np
import pytest

from gpu_util import same_bits, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _pinned(buf, torch):
    t = torch.from_numpy(np.ascontiguousarray(buf)).pin_memory()
    return t


CASES = [
    # ta, tb, m, n, k, alpha, beta, pad, form, rounding, panels
    ("N", "N", 700, 900, 500, complex(1.5, -0.5), complex(0.25, 0.75), 3, "fp32", "auto", 0),
    ("T", "C", 513, 1000, 257, complex(1, 0), complex(0, 0), 0, "fp32", "auto", 7),
    ("C", "T", 64, 2000, 3000, complex(0.5, 0.5), complex(-1, 0.5), 1, "fp32", "auto", 3),  # K split
    ("R", "N", 300, 40, 600, complex(1, 0), complex(0, 0), 0, "fp32", "auto", 0),
    ("N", "T", 1024, 1024, 1024, complex(1, 0), complex(0, 0), 0, "bf16x6", "off", 0),
    ("T", "N", 640, 1500, 512, complex(0.3, -0.7), complex(0.5, 0), 2, "tf32x3", "off", 5),
    ("N", "N", 2048, 2048, 2048, complex(1, 0), complex(0, 0), 0, "bf16x6", "auto", 0),  # rounding: one panel
    ("N", "C", 200, 300, 100, complex(0, 0), complex(0.5, -1.5), 1, "fp32", "auto", 0),  # alpha = 0
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}{c[1]}-{c[2]}x{c[3]}x{c[4]}-{c[8]}-p{c[10]}" for c in CASES])
def test_host_entry_equals_device_call(cg3m, oracle, cuda, h, case):
    import torch

    ta, tb, m, n, k, alpha, beta, pad, form, rounding, panels = case
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + pad, br + pad, m + pad
    a = oracle.make_matrix(ar, ac, lda, "UNIFORM_1", 11)
    b = oracle.make_matrix(br, bc, ldb, "UNIFORM_1", 12)
    c = oracle.make_matrix(m, n, ldc, "UNIFORM_1", 13)
    # device call
    C = to_dev(c, torch, cuda)
    dev_info = h.cgemm3m(ta, tb, m, n, k, alpha, to_dev(a, torch, cuda), lda, to_dev(b, torch, cuda), ldb, beta, C,
                         ldc, form=form, rounding=rounding)
    torch.cuda.synchronize()
    want = to_host(C)
    # host call
    Ah, Bh, Ch = _pinned(a, torch), _pinned(b, torch), _pinned(c, torch)
    info = h.cgemm3m_host(ta, tb, m, n, k, alpha, Ah, lda, Bh, ldb, beta, Ch, ldc, form=form, rounding=rounding,
                          panels=panels)
    got = Ch.numpy()
    assert same_bits(got, want), (case, dev_info, info)
    if alpha != 0:
        assert info["k_partitions"] == dev_info["k_partitions"]
        assert info["rounding"] == dev_info["rounding"]
    # padding rows of C untouched
    if pad:
        gv = got.reshape(n, ldc)[:, m:]
        cv = c.reshape(n, ldc)[:, m:]
        assert gv.tobytes() == cv.tobytes()


def test_host_entry_pageable_and_repeat(cg3m, oracle, cuda, h):
    """Pageable host memory works (without overlap), and repeated calls reuse the device copies."""
    import torch

    m, n, k = 333, 777, 222
    a = oracle.make_matrix(m, k, m, "UNIFORM_1", 21)
    b = oracle.make_matrix(k, n, k, "UNIFORM_1", 22)
    c0 = np.zeros(m * n, np.complex64)
    outs = []
    for _ in range(2):
        c = c0.copy()
        h.cgemm3m_host("N", "N", m, n, k, 1.0, torch.from_numpy(a), m, torch.from_numpy(b), k, 0.0,
                       torch.from_numpy(c), m)
        outs.append(c)
    assert outs[0].tobytes() == outs[1].tobytes()
    model = c0.copy()
    info = cg3m.plan("N", "N", m, n, k)
    oracle.cgemm3m_fp32_model("N", "N", m, n, k, 1.0 + 0j, a, m, b, k, 0j, model, m, span=info["k_span"])
    assert same_bits(outs[0], model)
