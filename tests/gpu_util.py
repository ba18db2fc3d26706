"""Helpers shared by the GPU tests: host<->device buffers, sub-problems for the
bit-exact model, NaN-aware bitwise comparison."""
import numpy as np


def to_dev(buf, torch, device):
    if buf is None:
        return None
    return torch.from_numpy(np.ascontiguousarray(buf)).to(device)


def to_host(t):
    return t.cpu().numpy()


def same_bits(x, y):
    """Bitwise equality of complex64 buffers, treating any NaN as equal to any NaN."""
    xf = np.ascontiguousarray(x).view(np.float32)
    yf = np.ascontiguousarray(y).view(np.float32)
    both_nan = np.isnan(xf) & np.isnan(yf)
    return bool(np.all((xf.view(np.uint32) == yf.view(np.uint32)) | both_nan))


def sub_problem(oracle, op, buf, ld, rows_of_op, cols_of_op, sel, axis):
    """Stored buffer of op(X) restricted to rows (axis=0) or columns (axis=1)
    of op(X), keeping the same op.  Returns (buffer, ld)."""
    sr, sc = oracle.stored_shape(op, rows_of_op, cols_of_op)
    X = oracle.unpack(buf, ld, sr, sc)
    normal = op in ("N", "R")
    # op(X) rows are stored rows when normal, stored columns otherwise.
    stored_axis = axis if normal else 1 - axis
    Y = X[sel, :] if stored_axis == 0 else X[:, sel]
    return np.ascontiguousarray(Y.T).reshape(-1).astype(np.complex64), Y.shape[0]


def run(cg3m_mod, h, torch, device, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, **kw):
    A = to_dev(a, torch, device)
    B = to_dev(b, torch, device)
    C = to_dev(c, torch, device)
    info = h.cgemm3m(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, **kw)
    torch.cuda.synchronize()
    return to_host(C), info
