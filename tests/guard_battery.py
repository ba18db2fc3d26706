"""Calls that together touch every workspace region of the cgemm3m paths
(packed planes, split partials, the rounding region with its exact-recompute
slices), used by test_gpu_guard_bands.py both with guard bands (in a child
process started with CG3M_GUARD_BANDS set) and without.  Returns a sha256
digest of each call's C."""
import hashlib

import numpy as np


def _square_mixed(oracle, n):
    a = oracle.make_matrix(n, n, n, "UNIFORM_1", 91)
    b = oracle.make_matrix(n, n, n, "UNIFORM_1", 92)
    A = a.reshape(n, n)
    B = b.reshape(n, n)
    for r in (5, 100, 777, 1500):
        A[:, r] *= np.float32(1024.0)
    for c in range(160, 166):
        B[c, :] *= np.float32(1024.0)
    return a, b


def run_battery(cg3m, oracle, torch, dev):
    h = cg3m.Handle(stream=torch.cuda.current_stream().cuda_stream)
    out = {}

    def dev_(x):
        return torch.from_numpy(np.ascontiguousarray(x)).to(dev)

    def call(name, ta, tb, m, n, k, alpha, beta, fill="UNIFORM_1", pad=0, **kw):
        ar, ac = oracle.stored_shape(ta, m, k)
        br, bc = oracle.stored_shape(tb, k, n)
        lda, ldb, ldc = ar + pad, br + pad, m + pad
        a = oracle.make_matrix(ar, ac, lda, fill, 11)
        b = oracle.make_matrix(br, bc, ldb, fill, 12)
        c = oracle.make_matrix(m, n, ldc, fill, 13)
        C = dev_(c)
        info = h.cgemm3m(ta, tb, m, n, k, alpha, dev_(a), lda, dev_(b), ldb, beta, C, ldc, **kw)
        torch.cuda.synchronize()
        out[name] = (hashlib.sha256(C.cpu().numpy().tobytes()).hexdigest(), info["path"], info["kernels"])

    call("fp32_512_cluster_split", "N", "N", 512, 512, 512, complex(1.5, -0.5), complex(0.25, 0.75))
    call("fp32_longk_merge_kernel", "N", "T", 64, 64, 16384, complex(0.5, 0.5), 0.0)
    call("fp32_ops_padded", "T", "C", 1000, 777, 3001, complex(0.7, 0.3), complex(-1.0, 0.5), pad=13)
    call("bf16x6_pair", "C", "N", 700, 600, 900, complex(0.7, 0.3), complex(-1.0, 0.5), form="bf16x6",
         engine="packed")
    call("tf32x3_forced_split", "N", "N", 300, 200, 4000, 1.0, 0.0, form="tf32x3", engine="packed",
         k_partitions=6)
    n = 2048
    a, b = _square_mixed(oracle, n)
    for form in ("fp32", "bf16x6"):
        C = torch.zeros(n * n, dtype=torch.complex64, device=dev)
        info = h.cgemm3m("N", "N", n, n, n, 1.0, dev_(a), n, dev_(b), n, 0.0, C, n, form=form)
        torch.cuda.synchronize()
        out[f"{form}_rounding_mixed"] = (hashlib.sha256(C.cpu().numpy().tobytes()).hexdigest(), info["rounding"],
                                         info["kernels"])
    pa = oracle.precision_matrix(n, n, 21)
    pb = oracle.precision_matrix(n, n, 22)
    for form in ("fp32", "bf16x6"):
        C = torch.zeros(n * n, dtype=torch.complex64, device=dev)
        info = h.cgemm3m("N", "N", n, n, n, 1.0, dev_(pa), n, dev_(pb), n, 0.0, C, n, form=form)
        torch.cuda.synchronize()
        out[f"{form}_rounding_dense"] = (hashlib.sha256(C.cpu().numpy().tobytes()).hexdigest(), info["rounding"],
                                         info["kernels"])
    return out
