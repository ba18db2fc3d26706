"""Python face of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only to check or to time the reference algorithm on the
host.  The product library never calls into it.

Provides
  * ctypes bindings to ``cg3m_oracle.c`` (reference-order cgemm, FP64 zgemm,
    the bit-exact plain-3M model and the rounding-correction restatement);
  * ``Cgemm3mComponentResult`` / ``verify_cgemm3m``: the reference's accuracy
    criterion (ops-blas/test/gemm/cgemm3m/cgemm3m_verify.h:22-84);
  * seeded fills for the reference's fill kinds and error norms vs FP64.
"""
from __future__ import annotations

import ctypes
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
import build_oracle as _build  # noqa: E402

OP = {"N": 0, "T": 1, "C": 2, "R": 3}
OP_NAMES = {0: "N", 1: "T", 2: "C", 3: "R"}

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        i = ctypes.c_int
        L.oracle_cgemm.argtypes = [i, i, i, i, i, P, P, i, P, i, P, P, i]
        L.oracle_zgemm.argtypes = [i, i, i, i, i, P, P, i, P, i, P, P, i, P]
        L.oracle_cgemm3m_fp32.argtypes = [i, i, i, i, i, P, P, i, P, i, P, P, i, i]
        L.oracle_cgemm_modes_fp32.argtypes = [i, i, i, i, i, i, i, P, P, i, P, i, P, P, i, i]
        L.oracle_risk_path.argtypes = [i, i, i, P, P, P, P]
        L.oracle_risk_path_rect.argtypes = [i, i, i, i, i, P, i, P, i, P, P]
        L.oracle_energy.argtypes = [i, i, i, P, i, P, i, P]
        L.oracle_select.argtypes = [i, P, P, P, ctypes.c_float, P]
        L.oracle_select.restype = ctypes.c_long
        L.oracle_recompute.argtypes = [i, i, i, P, i, P, i, P, P]
        L.oracle_recompute_dot.argtypes = [i, P, P, P]
        L.oracle_bridge.argtypes = [i]
        L.oracle_bridge.restype = ctypes.c_float
        L.oracle_segment_span.argtypes = [i]
        L.oracle_segment_span.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c64(x):
    return np.ascontiguousarray(x, dtype=np.complex64)


def _op(o):
    return OP[o] if isinstance(o, str) else int(o)


def stored_shape(op, rows_of_op, cols_of_op):
    """Stored (rows, cols) of X given op(X) is rows_of_op x cols_of_op."""
    return (rows_of_op, cols_of_op) if _op(op) in (0, 3) else (cols_of_op, rows_of_op)


def col_major_buffer(rows, cols, ld):
    """Flat complex64 buffer of ld*cols elements viewed column-major."""
    return np.zeros(max(1, ld * max(cols, 0)), dtype=np.complex64)


def cgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Reference-order FP32 cgemm in place on the flat column-major buffer ``c``."""
    al = np.array([alpha.real, alpha.imag], dtype=np.float32)
    be = np.array([beta.real, beta.imag], dtype=np.float32)
    a = _c64(a) if a is not None else None
    b = _c64(b) if b is not None else None
    assert c.dtype == np.complex64 and c.flags.c_contiguous
    lib().oracle_cgemm(_op(transa), _op(transb), m, n, k, _ptr(al), _ptr(a), lda, _ptr(b), ldb, _ptr(be), _ptr(c), ldc)
    return c


_timing_lib = None


def cgemm_timing(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """oracle_cgemm from the timing build (no volatile stores; same bytes)."""
    global _timing_lib
    if _timing_lib is None:
        lib()
        L = ctypes.CDLL(_build.LIB_TIMING)
        P, i = ctypes.c_void_p, ctypes.c_int
        L.oracle_cgemm.argtypes = [i, i, i, i, i, P, P, i, P, i, P, P, i]
        _timing_lib = L
    al = np.array([complex(alpha).real, complex(alpha).imag], np.float32)
    be = np.array([complex(beta).real, complex(beta).imag], np.float32)
    _timing_lib.oracle_cgemm(_op(transa), _op(transb), m, n, k, _ptr(al), _ptr(_c64(a)), lda, _ptr(_c64(b)), ldb,
                             _ptr(be), _ptr(c), ldc)
    return c


def zgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """FP64 product; returns an m x n complex128 array (column-major values)."""
    al = np.array([alpha.real, alpha.imag], dtype=np.float64)
    be = np.array([beta.real, beta.imag], dtype=np.float64)
    out = np.zeros(m * n, dtype=np.complex128)
    lib().oracle_zgemm(_op(transa), _op(transb), m, n, k, _ptr(al), _ptr(_c64(a)), lda, _ptr(_c64(b)), ldb,
                       _ptr(be), _ptr(_c64(c)), ldc, _ptr(out))
    return out.reshape(n, m).T


def zgemm_numpy(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """FP64 product through numpy (faster for large sizes); m x n complex128."""
    opa = op_matrix(a, lda, transa, m, k).astype(np.complex128)
    opb = op_matrix(b, ldb, transb, k, n).astype(np.complex128)
    out = complex(alpha) * (opa @ opb)
    if beta != 0:
        out = out + complex(beta) * unpack(c, ldc, m, n).astype(np.complex128)
    return out


def cgemm3m_fp32_model(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, span=0):
    """Bit-exact model of the plain FP32 3M GPU path (in place on ``c``)."""
    al = np.array([alpha.real, alpha.imag], dtype=np.float32)
    be = np.array([beta.real, beta.imag], dtype=np.float32)
    lib().oracle_cgemm3m_fp32(_op(transa), _op(transb), m, n, k, _ptr(al), _ptr(_c64(a)), lda, _ptr(_c64(b)), ldb,
                              _ptr(be), _ptr(c), ldc, int(span))
    return c


def cgemm_modes_model(mode, repair, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, span=0):
    """Bit-exact model of the on-chip product family (in place on ``c``):
    mode 0 = standard 3M, 1 = four products; ``repair`` recomputes non-finite
    products with the explicit four-product sum."""
    al = np.array([complex(alpha).real, complex(alpha).imag], dtype=np.float32)
    be = np.array([complex(beta).real, complex(beta).imag], dtype=np.float32)
    lib().oracle_cgemm_modes_fp32(int(mode), int(repair), _op(transa), _op(transb), m, n, k, _ptr(al), _ptr(_c64(a)),
                                  lda, _ptr(_c64(b)), ldb, _ptr(be), _ptr(c), ldc, int(span))
    return c


def risk_path(n, a, b, transa="N", transb="N"):
    """(path, C) of the unit-output square problem (lda = ldb = n), both column-major n x n."""
    path = np.zeros(n * n, dtype=np.float32)
    c = np.zeros(n * n, dtype=np.complex64)
    lib().oracle_risk_path(n, _op(transa), _op(transb), _ptr(_c64(a)), _ptr(_c64(b)), _ptr(path), _ptr(c))
    return path, c


def risk_path_rect(m, n, k, transa, a, lda, transb, b, ldb):
    """(path, C) of an m x n output block with full K, column-major (ld = m)."""
    path = np.zeros(m * n, dtype=np.float32)
    c = np.zeros(m * n, dtype=np.complex64)
    lib().oracle_risk_path_rect(m, n, k, _op(transa), _op(transb), _ptr(_c64(a)), lda, _ptr(_c64(b)), ldb,
                                _ptr(path), _ptr(c))
    return path, c


def select_flags(path, c, e_rows, e_cols, bridge_value, confidence=3.75):
    """Selection predicate elementwise in FP32 (same operations as oracle_select)."""
    f32 = np.float32
    c = np.asarray(c, np.complex64)
    mag = np.maximum(np.abs(c.real), np.abs(c.imag)).astype(f32)
    with np.errstate(over="ignore", invalid="ignore"):
        ee = (np.asarray(e_rows, f32)[:, None] * np.asarray(e_cols, f32)[None, :]).astype(f32)
        var = (f32(2.0 ** -48) * (np.asarray(path, f32) + (ee * f32(bridge_value)).astype(f32))).astype(f32)
        conf2 = f32(confidence) * f32(confidence)
        return (~np.isfinite(mag)) | (~np.isfinite(var)) | ((conf2 * var).astype(f32) >= f32(0.0001))


def energy(n, transa, transb, a, lda, b, ldb):
    e = np.zeros(2 * n, dtype=np.float32)
    lib().oracle_energy(n, _op(transa), _op(transb), _ptr(_c64(a)), lda, _ptr(_c64(b)), ldb, _ptr(e))
    return e


def select(n, c, e, path, confidence=3.75):
    flags = np.zeros(n * n, dtype=np.uint8)
    cnt = lib().oracle_select(n, _ptr(_c64(c)), _ptr(np.ascontiguousarray(e, np.float32)),
                              _ptr(np.ascontiguousarray(path, np.float32)), ctypes.c_float(confidence), _ptr(flags))
    return flags, int(cnt)


def recompute(n, transa, transb, a, lda, b, ldb, flags, c):
    lib().oracle_recompute(n, _op(transa), _op(transb), _ptr(_c64(a)), lda, _ptr(_c64(b)), ldb,
                           _ptr(np.ascontiguousarray(flags, np.uint8)), _ptr(c))
    return c


def recompute_dot(arow, bcol):
    out = np.zeros(2, dtype=np.float32)
    lib().oracle_recompute_dot(len(arow), _ptr(_c64(arow)), _ptr(_c64(bcol)), _ptr(out))
    return complex(out[0], out[1])


def bridge(n):
    return float(lib().oracle_bridge(n))


def segment_span(n):
    return int(lib().oracle_segment_span(n))


# --------------------------------------------------------------------------
# Layout helpers
# --------------------------------------------------------------------------

def unpack(buf, ld, rows, cols):
    """rows x cols matrix from a flat column-major buffer with leading dim ld."""
    if rows == 0 or cols == 0:
        return np.zeros((rows, cols), dtype=buf.dtype)
    return buf[: ld * cols].reshape(cols, ld)[:, :rows].T


def op_matrix(buf, ld, op, rows_of_op, cols_of_op):
    o = _op(op)
    sr, sc = stored_shape(o, rows_of_op, cols_of_op)
    x = unpack(buf, ld, sr, sc)
    if o in (1, 2):
        x = x.T
    if o in (2, 3):
        x = np.conj(x)
    return x


# --------------------------------------------------------------------------
# Fills (own definitions of the reference's fill kinds; the reference's
# generator lives in an unshipped fill.h, so values are this project's).
# --------------------------------------------------------------------------

FILL_KINDS = ("RANDOM_NORM_5_5", "VALUE_NORM_0", "VALUE_NORM_INF", "VALUE_NORM_NAN", "RANDOM_EXTREME",
              "RANDOM_ALTER", "NULLPTR", "UNIFORM_1")


def make_matrix(rows, cols, ld, fill, seed):
    """Flat column-major complex64 buffer (ld*cols) filled per ``fill``.

    RANDOM_NORM_5_5: real and imaginary parts uniform in [-5, 5].
    UNIFORM_1:       uniform in [-1, 1].
    VALUE_NORM_0/INF/NAN: every stored element (0,0) / (+inf,+inf) / (nan,nan).
    RANDOM_EXTREME:  random signs, magnitudes 2^e with e uniform in [-60, 60].
    RANDOM_ALTER:    uniform in [-5, 5] with alternating sign by linear index.
    Padding rows (ld > rows) hold a fixed sentinel so untouched padding is visible.
    NULLPTR returns None.
    """
    if fill == "NULLPTR":
        return None
    rng = np.random.default_rng(seed)
    size = max(1, ld * max(cols, 0))
    if fill in ("RANDOM_NORM_5_5", "RANDOM_ALTER"):
        re = rng.uniform(-5.0, 5.0, size)
        im = rng.uniform(-5.0, 5.0, size)
        if fill == "RANDOM_ALTER":
            sign = np.where(np.arange(size) % 2 == 0, 1.0, -1.0)
            re, im = np.abs(re) * sign, np.abs(im) * -sign
    elif fill == "UNIFORM_1":
        re = rng.uniform(-1.0, 1.0, size)
        im = rng.uniform(-1.0, 1.0, size)
    elif fill == "VALUE_NORM_0":
        re = np.zeros(size)
        im = np.zeros(size)
    elif fill == "VALUE_NORM_INF":
        re = np.full(size, np.inf)
        im = np.full(size, np.inf)
    elif fill == "VALUE_NORM_NAN":
        re = np.full(size, np.nan)
        im = np.full(size, np.nan)
    elif fill == "RANDOM_EXTREME":
        re = rng.choice([-1.0, 1.0], size) * np.exp2(rng.integers(-60, 61, size))
        im = rng.choice([-1.0, 1.0], size) * np.exp2(rng.integers(-60, 61, size))
    else:
        raise ValueError(fill)
    # assign the parts separately: re + 1j*im would turn an infinite imaginary
    # part into (nan, inf) through 0*inf
    out = np.empty(size, dtype=np.complex64)
    out.real = re
    out.imag = im
    if ld > rows and cols > 0:
        view = out[: ld * cols].reshape(cols, ld)
        view[:, rows:] = np.complex64(complex(-7.25, 3.5))
    return out


def precision_matrix(rows, cols, seed):
    """Precision-form workload data: Re ~ N(0,1); Im ~ N(0,1) * 2^e, e uniform
    integer in [-8, 8] drawn per column.  Contiguous column-major."""
    rng = np.random.default_rng(seed)
    re = rng.standard_normal((cols, rows))
    e = rng.integers(-8, 9, size=cols)
    im = rng.standard_normal((cols, rows)) * np.exp2(e)[:, None]
    return (re + 1j * im).astype(np.complex64).reshape(-1)


# --------------------------------------------------------------------------
# Verifier (ops-blas/test/gemm/cgemm3m/cgemm3m_verify.h:22-84)
# --------------------------------------------------------------------------

class Cgemm3mComponentResult:
    """Per-component (real or imag) accumulator of the reference criterion.

    A finite pair matches when |a-g| <= (1+|g|)/8192; the component passes when
    no non-finite pair failed, >= 99% of finite pairs matched, and the largest
    error is <= max(0.01, 32*ULP(g)) evaluated at the golden of the largest
    error.  Non-finite rules: NaN is equivalent to any non-finite; +/-inf must
    match exactly; finite vs non-finite fails.
    """

    def __init__(self):
        self.finite = 0
        self.matched = 0
        self.nonfinite = 0
        self.nonfinite_failed = 0
        self.max_error = 0.0
        self.max_error_limit = 0.01
        self.max_error_golden = 0.0

    def add(self, actual, golden):
        self.add_many(np.array([actual], np.float32), np.array([golden], np.float32))

    def add_many(self, actual, golden):
        actual = np.asarray(actual, np.float32).ravel()
        golden = np.asarray(golden, np.float32).ravel()
        fa, fg = np.isfinite(actual), np.isfinite(golden)
        nf = ~(fa & fg)
        if nf.any():
            a_nf, g_nf = actual[nf], golden[nf]
            both = ~np.isfinite(a_nf) & ~np.isfinite(g_nf)
            equiv = both & (np.isnan(a_nf) | np.isnan(g_nf) | (a_nf == g_nf))
            self.nonfinite += int(nf.sum())
            self.nonfinite_failed += int((~equiv).sum())
        fin = ~nf
        if fin.any():
            a = actual[fin].astype(np.float64)
            g = golden[fin].astype(np.float64)
            err = np.abs(a - g)
            self.finite += int(fin.sum())
            self.matched += int((err <= (1.0 + np.abs(g)) / 8192.0).sum())
            idx = int(np.argmax(err))
            if err[idx] > self.max_error:
                self.max_error = float(err[idx])
                gv = np.float32(g[idx])
                self.max_error_golden = float(gv)
                exponent = -126 if gv == 0 else max(-126, math.frexp(abs(float(gv)))[1] - 1)
                self.max_error_limit = max(0.01, 32.0 * math.ldexp(1.0, exponent - 23))

    def passed(self):
        return (self.nonfinite_failed == 0 and self.max_error <= self.max_error_limit
                and (self.finite == 0 or self.matched * 100 >= self.finite * 99))


def verify_cgemm3m(actual, golden, initial, m, n, ldc):
    """Reference verification of flat column-major buffers; returns (ok, real, imag, padding_ok)."""
    real, imag = Cgemm3mComponentResult(), Cgemm3mComponentResult()
    padding_ok = True
    if m > 0 and n > 0:
        A = actual[: ldc * n].reshape(n, ldc)
        G = golden[: ldc * n].reshape(n, ldc)
        I = initial[: ldc * n].reshape(n, ldc)
        real.add_many(A[:, :m].real, G[:, :m].real)
        imag.add_many(A[:, :m].imag, G[:, :m].imag)
        if ldc > m:
            padding_ok = A[:, m:].tobytes() == I[:, m:].tobytes()
    return real.passed() and imag.passed() and padding_ok, real, imag, padding_ok


def error_report(actual, exact):
    """Normwise and worst componentwise errors of an m x n result vs FP64.

    normwise = ||C - C64||_F / ||C64||_F; componentwise is reported for the real
    and imaginary parts separately as max |dX| / |X64| over elements with
    X64 != 0, plus the max absolute error per part.
    """
    actual = np.asarray(actual).astype(np.complex128)
    exact = np.asarray(exact).astype(np.complex128)
    diff = actual - exact
    denom = np.linalg.norm(exact)
    out = {"normwise": float(np.linalg.norm(diff) / denom) if denom > 0 else float(np.linalg.norm(diff))}
    for part, f in (("re", np.real), ("im", np.imag)):
        d = np.abs(f(diff))
        x = np.abs(f(exact))
        nz = x > 0
        out[f"comp_{part}"] = float((d[nz] / x[nz]).max()) if nz.any() else 0.0
        out[f"abs_{part}"] = float(d.max()) if d.size else 0.0
    return out
