"""cg3m -- Python face of the B200-native cgemm3m library (libcg3m.so).

The compute path is the C-ABI library built from ``../csrc`` for sm_100a; this
module only binds it with ctypes and passes device pointers from torch tensors.
There is no CPU or PyTorch fallback: if the library is missing, importing this
module raises.

Matrices follow the reference's conventions (ops-blas/include/cann_ops_blas.h
:497-500): column-major complex64, op in {N, T, C}, leading dimensions in
complex elements, alpha/beta complex scalars.  A column-major m x n matrix with
leading dimension ld is stored here as a torch complex64 tensor of shape
(n, ld) (row j = column j), or passed as any flat complex64 device buffer.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcg3m.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libcg3m.so not found at {LIB_PATH}; build it with "
        "`python ascend-open-source-contributions_b200/build_cg3m.py` (nvcc, sm_100a)")

_lib = ctypes.CDLL(LIB_PATH)

# ---- constants (include/cg3m.h) ------------------------------------------------
SUCCESS, HANDLE_IS_NULLPTR, INVALID_VALUE, INVALID_ENUM, ALLOC_FAILED, INTERNAL_ERROR, EXECUTION_FAILED, \
    NOT_SUPPORTED = range(8)
STATUS_NAMES = {0: "SUCCESS", 1: "HANDLE_IS_NULLPTR", 2: "INVALID_VALUE", 3: "INVALID_ENUM", 4: "ALLOC_FAILED",
                5: "INTERNAL_ERROR", 6: "EXECUTION_FAILED", 7: "NOT_SUPPORTED"}
OP = {"N": 0, "T": 1, "C": 2, "R": 3}
FORM = {"fp32": 0, "tf32x3": 1, "bf16x6": 2, "bf16x9": 3}
ROUNDING = {"auto": 0, "off": 1}
# FP32 engines: planner's choice, packed planes (pack + GEMM [+ merge]), one
# launch with the K partitions merged in a thread-block cluster.
ENGINE = {"auto": 0, "packed": 1, "onchip": 2}
# Tiles of the one-launch engine (onchip_tile - 1 indexes this list).
ONCHIP_TILES = [(128, 64), (64, 64), (128, 32), (32, 128), (64, 32), (32, 32)]


class cg3mComplex(ctypes.Structure):
    _fields_ = [("real", ctypes.c_float), ("imag", ctypes.c_float)]


class cg3mOptions(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int), ("rounding", ctypes.c_int), ("k_partitions", ctypes.c_int),
                ("tc_segment", ctypes.c_int), ("engine", ctypes.c_int), ("onchip_tile", ctypes.c_int),
                ("reserved", ctypes.c_int * 2)]


class cg3mCallInfo(ctypes.Structure):
    _fields_ = [("path", ctypes.c_int), ("form", ctypes.c_int), ("tile_m", ctypes.c_int), ("tile_n", ctypes.c_int),
                ("k_partitions", ctypes.c_int), ("k_span", ctypes.c_int), ("rounding", ctypes.c_int),
                ("kernels", ctypes.c_int), ("workspace_bytes", ctypes.c_size_t)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class cg3mProblem(ctypes.Structure):
    _fields_ = [("transa", ctypes.c_int), ("transb", ctypes.c_int), ("m", ctypes.c_int), ("n", ctypes.c_int),
                ("k", ctypes.c_int), ("alpha", cg3mComplex), ("beta", cg3mComplex), ("A", ctypes.c_void_p),
                ("lda", ctypes.c_int), ("B", ctypes.c_void_p), ("ldb", ctypes.c_int), ("C", ctypes.c_void_p),
                ("ldc", ctypes.c_int)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_CP = ctypes.POINTER(cg3mComplex)

SIGNATURES = {
    "cg3mCreate": [ctypes.POINTER(_P)],
    "cg3mDestroy": [_P],
    "cg3mSetStream": [_P, _P],
    "cg3mGetStream": [_P, ctypes.POINTER(_P)],
    "cg3mSetWorkspace": [_P, _P, ctypes.c_size_t],
    "cg3mGetVersion": [_P, ctypes.POINTER(_I)],
    "cg3mCgemm3m": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I],
    "cg3mCgemm3mEx": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I, ctypes.POINTER(cg3mOptions),
                      ctypes.POINTER(cg3mCallInfo)],
    "cg3mCgemm3mStridedBatched": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, ctypes.c_int64, _P, _I, ctypes.c_int64, _CP,
                                  _P, _I, ctypes.c_int64, _I],
    "cg3mCgemm": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I],
    "aclblasCgemm": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I],
    "cg3mCgemm3mHost": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I, ctypes.POINTER(cg3mOptions), _I,
                        ctypes.POINTER(cg3mCallInfo)],
    "cg3mBatchPlanCreate": [_P, ctypes.POINTER(cg3mProblem), _I, _I, ctypes.POINTER(_P), ctypes.POINTER(_I)],
    "cg3mBatchPlanExecute": [_P, _P, _I],
    "cg3mBatchPlanDestroy": [_P],
    "cg3mBatchPlanDescribe": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "cg3mGetDeviceStatus": [_P, ctypes.POINTER(_I)],
    "cg3mDiagFailAllocations": [_I],
    "cg3mDiagGuardStatus": [ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "cg3mGetRoundingStats": [_P, ctypes.POINTER(ctypes.c_longlong), _I],
    "cg3mDiagBoundedWait": [_P, ctypes.c_longlong, ctypes.POINTER(_I)],
    "cg3mCgemm3mNoAlloc": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I],
    "cg3mSetStageEvents": [_P, ctypes.POINTER(_P), _I],
    "cg3mValidate": [_I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I, _I, ctypes.POINTER(_I)],
    "cg3mPlan": [_I, _I, _I, _I, _I, _CP, _I, _I, _CP, _I, ctypes.POINTER(cg3mOptions), _I,
                 ctypes.POINTER(cg3mCallInfo)],
    "cg3mPlanOnchip": [_I, _I, _I, _I, _I, _I, ctypes.POINTER(cg3mCallInfo)],
    "cg3mZgemmReference": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I, _P],
    "cg3mErrorReport": [_P, _I, _I, _P, _I, _P, ctypes.POINTER(ctypes.c_double)],
    "aclblasCreate": [ctypes.POINTER(_P)],
    "aclblasDestroy": [_P],
    "aclblasSetStream": [_P, _P],
    "aclblasGetStream": [_P, ctypes.POINTER(_P)],
    "aclblasSetWorkspace": [_P, _P, ctypes.c_size_t],
    "aclblasGetVersion": [_P, ctypes.POINTER(_I)],
    "aclblasCgemm3m": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, _P, _I, _CP, _P, _I],
    "aclblasCgemm3mStridedBatched": [_P, _I, _I, _I, _I, _I, _CP, _P, _I, ctypes.c_int64, _P, _I, ctypes.c_int64,
                                     _CP, _P, _I, ctypes.c_int64, _I],
}

for _name, _args in SIGNATURES.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = ctypes.c_int

lib = _lib


def cx(z) -> cg3mComplex:
    z = complex(z)
    return cg3mComplex(z.real, z.imag)


def _op(o):
    return OP[o] if isinstance(o, str) else int(o)


class Cg3mError(RuntimeError):
    def __init__(self, status, what=""):
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}")
        self.status = status


def _check(status, what):
    if status != SUCCESS:
        raise Cg3mError(status, what)


def ptr(t):
    """Device (or host) address of a torch tensor / None."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


class Handle:
    """Owns one cg3m handle bound to a CUDA stream (default: torch's current)."""

    def __init__(self, stream=None):
        self.h = ctypes.c_void_p()
        _check(_lib.cg3mCreate(ctypes.byref(self.h)), "cg3mCreate")
        if stream is not None:
            self.set_stream(stream)

    def set_stream(self, stream):
        s = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream)
        _check(_lib.cg3mSetStream(self.h, ctypes.c_void_p(s)), "cg3mSetStream")

    def close(self):
        if self.h:
            _lib.cg3mDestroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stage_events(self, events):
        """Record the given torch.cuda.Event objects around each kernel of later
        calls: kernel j between events[2j] and events[2j + 1]."""
        for e in events:
            if not e.cuda_event:  # torch creates the CUDA event lazily on first record
                e.record()
        arr = (ctypes.c_void_p * max(1, len(events)))(*[ctypes.c_void_p(e.cuda_event) for e in events])
        _check(_lib.cg3mSetStageEvents(self.h, arr, len(events)), "cg3mSetStageEvents")

    def device_status(self):
        f = ctypes.c_int()
        _check(_lib.cg3mGetDeviceStatus(self.h, ctypes.byref(f)), "cg3mGetDeviceStatus")
        return f.value

    def rounding_stats(self):
        """Counters of the last call's rounding pass (synchronizes): flagged
        outputs, those recomputed by the tile kernels and those recomputed one
        by one; None when the last call ran no rounding pass."""
        v = (ctypes.c_longlong * 6)()
        _check(_lib.cg3mGetRoundingStats(self.h, v, 6), "cg3mGetRoundingStats")
        if v[0] < 0:
            return None
        return {"flagged": v[0], "dense_outputs": v[1], "sparse_outputs": v[2], "fallback_outputs": v[3],
                "exact_tiles": v[4], "exact_positions": v[5]}

    def cgemm3m(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, form="fp32", rounding="auto",
                k_partitions=0, raw=False, tc_segment=0, engine="auto", onchip_tile=0):
        """C <- alpha*op(A)*op(B) + beta*C on device buffers; returns the call info.

        ``raw=True`` calls the drop-in cg3mCgemm3m (FP32 form only) and returns
        the status instead of raising.  ``engine`` ("auto", "packed", "onchip")
        and ``onchip_tile`` (0 or 1..6, see ONCHIP_TILES) pick the FP32 engine."""
        al, be = cx(alpha), cx(beta)
        if raw:
            return _lib.cg3mCgemm3m(self.h, _op(transa), _op(transb), m, n, k, ctypes.byref(al), ptr(A), lda, ptr(B),
                                    ldb, ctypes.byref(be), ptr(C), ldc)
        opts = cg3mOptions(FORM[form] if isinstance(form, str) else form,
                           ROUNDING[rounding] if isinstance(rounding, str) else rounding, k_partitions, tc_segment,
                           ENGINE[engine] if isinstance(engine, str) else engine, onchip_tile)
        info = cg3mCallInfo()
        st = _lib.cg3mCgemm3mEx(self.h, _op(transa), _op(transb), m, n, k, ctypes.byref(al), ptr(A), lda, ptr(B), ldb,
                                ctypes.byref(be), ptr(C), ldc, ctypes.byref(opts), ctypes.byref(info))
        _check(st, "cg3mCgemm3mEx")
        return info.as_dict()

    def cgemm(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        """cg3mCgemm (the reference's aclblasCgemm); returns the status."""
        al, be = cx(alpha), cx(beta)
        return _lib.cg3mCgemm(self.h, _op(transa), _op(transb), m, n, k, ctypes.byref(al), ptr(A), lda, ptr(B), ldb,
                              ctypes.byref(be), ptr(C), ldc)

    def cgemm3m_strided_batched(self, transa, transb, m, n, k, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC,
                                batch):
        """cg3mCgemm3mStridedBatched on device buffers; returns the status."""
        al, be = cx(alpha), cx(beta)
        return _lib.cg3mCgemm3mStridedBatched(self.h, _op(transa), _op(transb), m, n, k, ctypes.byref(al), ptr(A),
                                              lda, sA, ptr(B), ldb, sB, ctypes.byref(be), ptr(C), ldc, sC, batch)

    def cgemm3m_host(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, form="fp32",
                     rounding="auto", k_partitions=0, tc_segment=0, panels=0):
        """cg3mCgemm3mHost: A, B, C are HOST buffers (page-locked torch CPU
        tensors overlap best); copies and panels are pipelined inside the
        call, which returns with C on the host.  Returns the call info."""
        al, be = cx(alpha), cx(beta)
        opts = cg3mOptions(FORM[form] if isinstance(form, str) else form,
                           ROUNDING[rounding] if isinstance(rounding, str) else rounding, k_partitions, tc_segment)
        info = cg3mCallInfo()
        st = _lib.cg3mCgemm3mHost(self.h, _op(transa), _op(transb), m, n, k, ctypes.byref(al), _addr(A), lda,
                                  _addr(B), ldb, ctypes.byref(be), _addr(C), ldc, ctypes.byref(opts), int(panels),
                                  ctypes.byref(info))
        _check(st, "cg3mCgemm3mHost")
        return info.as_dict()

    def batch_plan(self, problems, tune=True):
        """Plan a heterogeneous batch (one persistent launch per execute).

        ``problems``: sequence of (transa, transb, m, n, k, alpha, A, lda, B,
        ldb, beta, C, ldc) with device buffers (torch tensors or addresses).
        The buffers must stay alive while the plan is used."""
        return BatchPlan(self, problems, tune)

    def zgemm_reference(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, out64):
        al, be = cx(alpha), cx(beta)
        _check(_lib.cg3mZgemmReference(self.h, _op(transa), _op(transb), m, n, k, ctypes.byref(al), ptr(A), lda,
                                       ptr(B), ldb, ctypes.byref(be), ptr(C), ldc, ptr(out64)), "cg3mZgemmReference")

    def error_report(self, m, n, C, ldc, out64):
        rep = (ctypes.c_double * 5)()
        _check(_lib.cg3mErrorReport(self.h, m, n, ptr(C), ldc, ptr(out64), rep), "cg3mErrorReport")
        return {"normwise": rep[0], "comp_re": rep[1], "comp_im": rep[2], "abs_re": rep[3], "abs_im": rep[4]}


def _addr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    return ctypes.c_void_p(x.data_ptr())


class BatchPlan:
    """cg3mBatchPlan: the batch's tile/K-split tables and device task list."""

    def __init__(self, handle, problems, tune=True):
        self.handle = handle
        self._keep = list(problems)  # buffers referenced by the plan
        arr = (cg3mProblem * max(1, len(problems)))()
        for i, (ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc) in enumerate(problems):
            arr[i] = cg3mProblem(_op(ta), _op(tb), m, n, k, cx(alpha), cx(beta), _addr(A), lda, _addr(B), ldb,
                                 _addr(C), ldc)
        self.count = len(problems)
        self.p = ctypes.c_void_p()
        bad = ctypes.c_int(-1)
        st = _lib.cg3mBatchPlanCreate(handle.h, arr, self.count, int(bool(tune)), ctypes.byref(self.p),
                                      ctypes.byref(bad))
        if st != SUCCESS:
            err = Cg3mError(st, f"cg3mBatchPlanCreate (problem {bad.value})")
            err.bad_index = bad.value
            raise err

    def execute(self, use_graph=True):
        _check(_lib.cg3mBatchPlanExecute(self.handle.h, self.p, int(bool(use_graph))), "cg3mBatchPlanExecute")

    def describe(self):
        """Per problem: (tile_m, tile_n, k_partitions); zeros for quick returns."""
        n = max(1, self.count)
        tm, tn, kp = (ctypes.c_int * n)(), (ctypes.c_int * n)(), (ctypes.c_int * n)()
        _check(_lib.cg3mBatchPlanDescribe(self.p, tm, tn, kp), "cg3mBatchPlanDescribe")
        return [(tm[i], tn[i], kp[i]) for i in range(self.count)]

    def close(self):
        if self.p:
            _lib.cg3mBatchPlanDestroy(self.p)
            self.p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, allow_conj_only=False):
    """Host-only validation (no device access): (status, action)."""
    act = ctypes.c_int()
    al = ctypes.byref(cx(alpha)) if alpha is not None else None
    be = ctypes.byref(cx(beta)) if beta is not None else None
    st = _lib.cg3mValidate(_op(transa), _op(transb), m, n, k, al, A, lda, B, ldb, be, C, ldc, int(allow_conj_only),
                           ctypes.byref(act))
    return st, act.value


def plan(transa, transb, m, n, k, alpha=1, beta=0, lda=None, ldb=None, ldc=None, form="fp32", rounding="auto",
         k_partitions=0, sm_count=148, engine="auto", onchip_tile=0):
    """The planner's decision (host only)."""
    ta, tb = _op(transa), _op(transb)
    lda = lda or (m if ta in (0, 3) else k)
    ldb = ldb or (k if tb in (0, 3) else n)
    ldc = ldc or m
    opts = cg3mOptions(FORM[form], ROUNDING[rounding], k_partitions, 0,
                       ENGINE[engine] if isinstance(engine, str) else engine, onchip_tile)
    info = cg3mCallInfo()
    _check(_lib.cg3mPlan(ta, tb, m, n, k, ctypes.byref(cx(alpha)), lda, ldb, ctypes.byref(cx(beta)), ldc,
                         ctypes.byref(opts), sm_count, ctypes.byref(info)), "cg3mPlan")
    return info.as_dict()


def stage_names(info):
    """Names of the kernels one call launched, in launch order, from its call
    info (the order cg3mSetStageEvents records them in)."""
    k = int(info["kernels"])
    if info["path"] == 4:
        return ["onchip"][:k]
    if info["rounding"]:
        fp32 = info["form"] == FORM["fp32"]
        if fp32:
            names = ["pack", "gemm_path", "pack_rows", "energy", "select", "replay_tiles", "lanes_needed",
                     "lane_major", "replay_outputs"]
        else:
            # packed rows with the leading planes and the energies first; the
            # risk-plane GEMM selects; the rest of the planes only for the bands
            # the form's products read
            names = ["pack_rows", "energy", "gemm_path", "exact_split", "band_need", "pack_rest",
                     "gemm_form_tiles", "exact_tiles", "exact_crt", "lanes_needed", "lane_major",
                     "recompute_fp64_outputs", "fallback_fp64"]
    else:
        names = ["pack", "gemm", "merge"]
    names = names[:k]
    return names + [f"kernel{i}" for i in range(len(names), k)]


def plan_onchip(m, n, k, mode=0, batch=1, sm_count=148):
    """The on-chip family's plan (cg3mCgemm / strided batches), host only."""
    info = cg3mCallInfo()
    _check(_lib.cg3mPlanOnchip(m, n, k, int(mode), int(batch), int(sm_count), ctypes.byref(info)), "cg3mPlanOnchip")
    return info.as_dict()


_default_handles = {}


def default_handle():
    """A per-process handle following torch's current stream."""
    import torch

    dev = torch.cuda.current_device()
    h = _default_handles.get(dev)
    if h is None:
        h = _default_handles[dev] = Handle()
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    return h


def cgemm3m(A, B, transa="N", transb="N", alpha=1.0, beta=0.0, C=None, form="fp32", rounding="auto"):
    """Convenience wrapper on torch complex64 tensors in *row-major torch* shape.

    ``A`` holds op-stored matrix X as a torch (rows, cols) tensor; it is handed
    to the library as the column-major matrix X^T (no copy), so this computes
    the same product torch would: result = alpha*opt(A) @ opt(B) + beta*C where
    opt() applies ``transa``/``transb`` to the torch matrices.  Returns C.
    """
    import torch

    if not (A.is_cuda and B.is_cuda):
        raise ValueError("cg3m runs on CUDA tensors only")
    A = A.contiguous()
    B = B.contiguous()
    ta, tb = _op(transa), _op(transb)
    ar, ac = A.shape
    br, bc = B.shape
    m, k = (ar, ac) if ta in (0, 3) else (ac, ar)
    k2, n = (br, bc) if tb in (0, 3) else (bc, br)
    if k != k2:
        raise ValueError("inner dimensions differ")
    # torch row-major (rows, cols) == column-major (cols, rows): compute
    # C^T = op(B)^T op(A)^T, i.e. swap the operands (the reference's C^T
    # convention, gemm_host_common.h:69-74).
    if C is None:
        C = torch.zeros((m, n), dtype=torch.complex64, device=A.device)
    else:
        C = C.contiguous()
    h = default_handle()
    h.cgemm3m(tb, ta, n, m, k, alpha, B, bc, A, ac, beta, C, n, form=form, rounding=rounding)
    return C
