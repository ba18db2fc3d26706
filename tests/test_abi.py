"""CPU tests of the C-ABI library: it loads, exports every declared symbol, and
its host logic (validation order, statuses, quick returns, handle semantics,
planner) behaves as the reference's -- all without touching a GPU.

Reference: ValidateCgemmParams / LaunchComplexGemm (ops-blas/blas/gemm/arch35/
cgemm_host.cpp:589-634,687-730), handle API (ops-blas/include/cann_ops_blas.h
:31-110), ED contract rows of cgemm3m_test.csv (TC_ED_306-337).
"""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in ("cg3m.h", "cg3m_aclblas.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b((?:cg3m|aclblas)[A-Za-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_library_exports_every_declared_symbol(cg3m):
    names = declared_functions()
    assert "cg3mCgemm3m" in names and "aclblasCgemm3m" in names
    for n in names:
        assert hasattr(cg3m.lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", cg3m.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    for n in names:
        assert n in exported, n
    # nothing but the C ABI is exported
    assert all(s.startswith(("cg3m", "aclblas")) for s in exported if not s.startswith("_"))


def test_no_cpu_fallback_symbols(cg3m):
    """The library links no BLAS and carries no host GEMM: only CUDA kernels compute."""
    out = subprocess.run(["nm", "-D", "--undefined-only", cg3m.LIB_PATH], capture_output=True, text=True).stdout
    assert "gemm_" not in out and "cblas" not in out


# ---------------------------------------------------------------- handle API

def test_handle_lifecycle(cg3m):
    L = cg3m.lib
    h = ctypes.c_void_p()
    assert L.cg3mCreate(None) == cg3m.HANDLE_IS_NULLPTR
    assert L.cg3mCreate(ctypes.byref(h)) == cg3m.SUCCESS and h.value
    again = ctypes.c_void_p(h.value)
    assert L.cg3mCreate(ctypes.byref(again)) == cg3m.INVALID_VALUE  # *handle must be null
    s = ctypes.c_void_p()
    assert L.cg3mGetStream(h, ctypes.byref(s)) == cg3m.SUCCESS and not s.value
    assert L.cg3mGetStream(h, None) == cg3m.INVALID_VALUE
    assert L.cg3mSetStream(None, None) == cg3m.HANDLE_IS_NULLPTR
    assert L.cg3mSetWorkspace(h, None, 16) == cg3m.INVALID_VALUE
    assert L.cg3mSetWorkspace(h, ctypes.c_void_p(0x1000), 0) == cg3m.INVALID_VALUE
    v = ctypes.c_int()
    assert L.cg3mGetVersion(None, ctypes.byref(v)) == cg3m.SUCCESS and v.value == 10000
    assert L.cg3mGetVersion(h, None) == cg3m.INVALID_VALUE
    flags = ctypes.c_int(7)
    assert L.cg3mGetDeviceStatus(h, ctypes.byref(flags)) == cg3m.SUCCESS and flags.value == 0
    assert L.cg3mDestroy(h) == cg3m.SUCCESS
    assert L.cg3mDestroy(None) == cg3m.HANDLE_IS_NULLPTR


def test_aclblas_names_bind_the_same_handles(cg3m):
    L = cg3m.lib
    h = ctypes.c_void_p()
    assert L.aclblasCreate(ctypes.byref(h)) == cg3m.SUCCESS
    one, zero = cg3m.cx(1), cg3m.cx(0)
    assert L.aclblasCgemm3m(None, 0, 0, 0, 0, 0, ctypes.byref(one), None, 1, None, 1, ctypes.byref(zero), None,
                            1) == cg3m.HANDLE_IS_NULLPTR
    assert L.aclblasCgemm3m(h, 0, 0, 0, 3, 2, ctypes.byref(one), None, 1, None, 2, ctypes.byref(zero), None,
                            1) == cg3m.SUCCESS
    assert L.aclblasDestroy(h) == cg3m.SUCCESS


# ---------------------------------------------------------------- validation

def _case_args(c, cg3m):
    ta = 999 if c["transa"] == 999 else cg3m.OP[c["transa"]]
    tb = 999 if c["transb"] == 999 else cg3m.OP[c["transb"]]
    alpha = None if c["alpha"][0] is None else complex(c["alpha"][0], c["alpha"][1])
    beta = None if c["beta"][0] is None else complex(c["beta"][0], c["beta"][1])
    dummy = ctypes.c_void_p(0x1000)  # never dereferenced on these paths
    A = None if c["a_fill"] == "NULLPTR" else dummy
    B = None if c["b_fill"] == "NULLPTR" else dummy
    C = None if c["c_fill"] == "NULLPTR" else dummy
    return ta, tb, alpha, beta, A, B, C


def test_contract_rows_statuses(cg3m, cases):
    """Every row of the reference's case table gets the expected status from the
    host-only validator, and the ED rows also from the drop-in entry itself
    when the call needs no device."""
    h = cg3m.Handle()
    checked = 0
    for c in cases["cases"]:
        ta, tb, alpha, beta, A, B, C = _case_args(c, cg3m)
        st, action = cg3m.validate(ta, tb, c["m"], c["n"], c["k"], alpha, A, c["lda"], B, c["ldb"], beta, C, c["ldc"])
        expect = getattr(cg3m, c["expect"])
        assert st == expect, c["name"]
        if st != cg3m.SUCCESS or action == 0:
            al = ctypes.byref(cg3m.cx(alpha)) if alpha is not None else None
            be = ctypes.byref(cg3m.cx(beta)) if beta is not None else None
            got = cg3m.lib.cg3mCgemm3m(h.h, ta, tb, c["m"], c["n"], c["k"], al, A, c["lda"], B, c["ldb"], be, C,
                                       c["ldc"])
            assert got == expect, c["name"]
            checked += 1
    assert checked >= 16


@pytest.mark.parametrize("m,n,k,beta,action", [
    (0, 16, 16, 0, 0), (16, 0, 16, 0, 0), (16, 16, 0, 1, 0), (16, 16, 0, 0, 1), (16, 16, 0, 0.5, 1),
    (16, 16, 16, 0, 2),
])
def test_quick_return_classification(cg3m, m, n, k, beta, action):
    dummy = ctypes.c_void_p(0x1000)
    st, act = cg3m.validate("N", "N", m, n, k, 1.0, dummy, max(1, m), dummy, max(1, k), beta, dummy, max(1, m))
    assert st == cg3m.SUCCESS and act == action


def test_alpha_zero_allows_null_inputs(cg3m):
    dummy = ctypes.c_void_p(0x1000)
    st, act = cg3m.validate("N", "N", 3, 2, 7, 0.0, None, 3, None, 7, complex(0.5, -0.25), dummy, 5)
    assert st == cg3m.SUCCESS and act == 1
    st, _ = cg3m.validate("N", "N", 3, 2, 7, 1.0, None, 3, None, 7, 0.0, dummy, 5)
    assert st == cg3m.INVALID_VALUE


def test_conj_only_op_is_extension_only(cg3m):
    dummy = ctypes.c_void_p(0x1000)
    st, _ = cg3m.validate("R", "N", 4, 4, 4, 1.0, dummy, 4, dummy, 4, 0.0, dummy, 4)
    assert st == cg3m.INVALID_VALUE
    st, act = cg3m.validate("R", "R", 4, 4, 4, 1.0, dummy, 4, dummy, 4, 0.0, dummy, 4, allow_conj_only=True)
    assert st == cg3m.SUCCESS and act == 2


def test_validation_order(cg3m):
    """Enum before dims before ld before scalars before pointers (cgemm_host.cpp:589-634)."""
    dummy = ctypes.c_void_p(0x1000)
    assert cg3m.validate(999, "N", -1, 4, 4, None, None, 0, None, 0, None, None, 0)[0] == cg3m.INVALID_VALUE
    # bad ld is an error even for an empty output
    assert cg3m.validate("N", "N", 0, 4, 4, 1.0, None, 0, None, 4, 0.0, None, 1)[0] == cg3m.INVALID_VALUE
    # null scalars are errors even for an empty output
    assert cg3m.validate("N", "N", 0, 4, 4, None, None, 1, None, 4, 0.0, None, 1)[0] == cg3m.INVALID_VALUE
    # an empty output needs no matrices at all
    assert cg3m.validate("N", "N", 0, 4, 4, 1.0, None, 1, None, 4, 0.0, None, 1) == (cg3m.SUCCESS, 0)
    assert cg3m.validate("T", "N", 4, 4, 8, 1.0, dummy, 7, dummy, 8, 0.0, dummy, 4)[0] == cg3m.INVALID_VALUE


def test_strided_batched_statuses_without_device(cg3m):
    L = cg3m.lib
    h = cg3m.Handle()
    one, zero = ctypes.byref(cg3m.cx(1)), ctypes.byref(cg3m.cx(0))
    assert L.cg3mCgemm3mStridedBatched(None, 0, 0, 2, 2, 2, one, None, 2, 4, None, 2, 4, zero, None, 2, 4,
                                       1) == cg3m.HANDLE_IS_NULLPTR
    assert L.cg3mCgemm3mStridedBatched(h.h, 999, 0, 2, 2, 2, one, None, 2, 4, None, 2, 4, zero, None, 2, 4,
                                       1) == cg3m.INVALID_ENUM
    assert L.cg3mCgemm3mStridedBatched(h.h, 0, 0, 2, 2, 2, one, None, 2, 4, None, 2, 4, zero, None, 2, 4,
                                       -1) == cg3m.INVALID_VALUE
    assert L.cg3mCgemm3mStridedBatched(h.h, 0, 0, 2, 2, 2, one, None, 2, 4, None, 2, 4, zero, None, 2, 4,
                                       0) == cg3m.SUCCESS
    assert L.cg3mCgemm3mStridedBatched(h.h, 0, 0, 2, 2, 2, None, None, 2, 4, None, 2, 4, zero, None, 2, 4,
                                       0) == cg3m.INVALID_VALUE


# ---------------------------------------------------------------- planner

def test_planner_large_square_is_single_partition(cg3m):
    p = cg3m.plan("N", "N", 4096, 4096, 4096)
    assert p["k_partitions"] == 1 and (p["tile_m"], p["tile_n"]) == (128, 64)
    assert p["k_span"] == 4096


def test_planner_long_k_few_tiles_splits_k(cg3m):
    p = cg3m.plan("N", "N", 128, 128, 65536, alpha=complex(0.7, 0.3), beta=complex(-1, 0.5))
    assert p["k_partitions"] > 1
    assert p["k_span"] % 16 == 0
    assert (p["k_partitions"] - 1) * p["k_span"] < 65536 <= p["k_partitions"] * p["k_span"]


def test_planner_narrow_long_k_forces_eight_parts(cg3m):
    p = cg3m.plan("N", "N", 8, 16, 4096)
    assert p["k_partitions"] >= 8


def test_planner_forced_partitions(cg3m):
    p = cg3m.plan("N", "N", 300, 200, 1000, k_partitions=3)
    assert p["k_partitions"] == 3 and p["k_span"] == 336


def test_planner_onchip_engine(cg3m):
    """Engine 2 (one launch, cluster-merged K partitions): no workspace, one
    kernel, at most 8 partitions; refused for the tensor-core forms, with the
    rounding pass, beyond 8 partitions, and for unknown engines or tiles."""
    p = cg3m.plan("N", "N", 300, 200, 1000, engine="onchip", onchip_tile=2, k_partitions=5)
    assert p["path"] == 4 and p["kernels"] == 1 and p["workspace_bytes"] == 0
    assert (p["tile_m"], p["tile_n"]) == (64, 64) and p["k_partitions"] == 5 and p["k_span"] == 208
    p = cg3m.plan("N", "N", 300, 200, 40, engine="onchip", k_partitions=8)
    assert p["k_partitions"] == 3 and p["k_span"] == 16  # the last partition must be non-empty
    for kw in ({"form": "bf16x6"}, {"k_partitions": 9}, {"onchip_tile": 7}):
        with pytest.raises(cg3m.Cg3mError):
            cg3m.plan("N", "N", 300, 200, 1000, engine="onchip", **kw)
    with pytest.raises(cg3m.Cg3mError):
        cg3m.plan("N", "N", 2048, 2048, 2048, engine="onchip")  # the rounding pass needs the packed engine
    with pytest.raises(cg3m.Cg3mError):
        cg3m.plan("N", "N", 300, 200, 1000, engine=3)
    assert cg3m.plan("N", "N", 300, 200, 1000, engine="packed", k_partitions=5)["path"] == 3
    # small tensor-core calls run as the plain FP32 one-launch product unless forced
    small = cg3m.plan("N", "N", 128, 128, 128, form="bf16x6", rounding="off")
    assert small["form"] == cg3m.FORM["fp32"] and small["path"] == 4
    forced = cg3m.plan("N", "N", 128, 128, 128, form="bf16x6", rounding="off", engine="packed")
    assert forced["form"] == cg3m.FORM["bf16x6"] and forced["path"] in (2, 3)
    big = cg3m.plan("N", "N", 4096, 4096, 4096, form="bf16x6", rounding="off")
    assert big["form"] == cg3m.FORM["bf16x6"]


def test_rounding_gate(cg3m):
    """The pass runs exactly for square contiguous unit-output orders 2048..4096."""
    assert cg3m.plan("N", "N", 2048, 2048, 2048)["rounding"] == 1
    assert cg3m.plan("C", "T", 4096, 4096, 4096)["rounding"] == 1
    assert cg3m.plan("N", "N", 2047, 2047, 2047)["rounding"] == 0
    assert cg3m.plan("N", "N", 4097, 4097, 4097)["rounding"] == 0
    assert cg3m.plan("N", "N", 2048, 2048, 2048, alpha=complex(1, 0.5))["rounding"] == 0
    assert cg3m.plan("N", "N", 2048, 2048, 2048, beta=0.5)["rounding"] == 0
    assert cg3m.plan("N", "N", 2048, 2048, 2048, lda=2050)["rounding"] == 0
    assert cg3m.plan("N", "N", 2048, 2048, 2048, rounding="off")["rounding"] == 0


def test_tc_rounding_pass_runs_unsplit(cg3m):
    """A requested K split does not reach the tensor-core forms' rounding pass,
    whose risk plane and form products run over the whole K; with the pass off
    (or for the FP32 form, whose split is part of the reference's arithmetic)
    the request stands."""
    for form in ("tf32x3", "bf16x6", "bf16x9"):
        on = cg3m.plan("N", "N", 2048, 2048, 2048, form=form, k_partitions=4)
        assert on["rounding"] == 1 and on["k_partitions"] == 1
        off = cg3m.plan("N", "N", 2048, 2048, 2048, form=form, k_partitions=4, rounding="off")
        assert off["k_partitions"] == 4
    fp32 = cg3m.plan("N", "N", 2048, 2048, 2048, form="fp32", k_partitions=4)
    assert fp32["rounding"] == 1 and fp32["k_partitions"] == 4


def test_rounding_stage_names_match_kernel_count(cg3m):
    """The names cg3mSetStageEvents' brackets are reported under cover exactly
    the kernels a rounding call launches: the FP32 form's pack, path GEMM and
    replay (9), the tensor-core forms' packed rows with the leading planes and
    the energies first, the selection inside the risk-plane GEMM and the banded
    rest of the planes after it (13)."""
    fp32 = cg3m.plan("N", "N", 4096, 4096, 4096, form="fp32")
    names = cg3m.stage_names(fp32)
    assert fp32["kernels"] == 9 and len(names) == 9 and names[:2] == ["pack", "gemm_path"]
    for form in ("tf32x3", "bf16x6", "bf16x9"):
        tc = cg3m.plan("N", "N", 4096, 4096, 4096, form=form)
        names = cg3m.stage_names(tc)
        assert tc["kernels"] == 13 and len(names) == 13, (form, tc, names)
        assert names[:3] == ["pack_rows", "energy", "gemm_path"] and "kernel" not in "".join(names)
        assert "select" not in names
        assert names.index("band_need") < names.index("pack_rest") < names.index("gemm_form_tiles")


def test_batch_plan_validation_without_device(cg3m):
    """Argument errors of cg3mBatchPlanCreate come from the host-side
    validation, per problem in order, before any device work."""
    L = cg3m.lib
    h = cg3m.Handle()
    plan = ctypes.c_void_p()
    bad = ctypes.c_int(-1)
    arr = (cg3m.cg3mProblem * 3)()
    dummy = ctypes.c_void_p(0x1000)
    for i in range(3):
        arr[i] = cg3m.cg3mProblem(0, 0, 4, 4, 4, cg3m.cx(1), cg3m.cx(0), dummy, 4, dummy, 4, dummy, 4)
    arr[1].lda = 2  # lda < m
    assert L.cg3mBatchPlanCreate(None, arr, 3, 0, ctypes.byref(plan), ctypes.byref(bad)) == cg3m.HANDLE_IS_NULLPTR
    assert L.cg3mBatchPlanCreate(h.h, arr, -1, 0, ctypes.byref(plan), ctypes.byref(bad)) == cg3m.INVALID_VALUE
    assert L.cg3mBatchPlanCreate(h.h, None, 3, 0, ctypes.byref(plan), ctypes.byref(bad)) == cg3m.INVALID_VALUE
    assert L.cg3mBatchPlanCreate(h.h, arr, 3, 0, None, ctypes.byref(bad)) == cg3m.INVALID_VALUE
    assert L.cg3mBatchPlanCreate(h.h, arr, 3, 0, ctypes.byref(plan), ctypes.byref(bad)) == cg3m.INVALID_VALUE
    assert bad.value == 1 and not plan.value
    arr[1].lda = 4
    arr[2].transb = 7  # an unknown op: the single call's status
    assert L.cg3mBatchPlanCreate(h.h, arr, 3, 0, ctypes.byref(plan), ctypes.byref(bad)) == cg3m.validate(
        "N", 7, 4, 4, 4, 1.0, 0x1000, 4, 0x1000, 4, 0.0, 0x1000, 4)[0] == cg3m.INVALID_VALUE
    assert bad.value == 2
    # op code R is accepted in a batch (the differentiable form's conj-only op)
    arr[2].transb = 3
    arr[0].C = None
    assert L.cg3mBatchPlanCreate(h.h, arr, 3, 0, ctypes.byref(plan), ctypes.byref(bad)) == cg3m.INVALID_VALUE
    assert bad.value == 0
    assert L.cg3mBatchPlanExecute(None, None, 0) == cg3m.HANDLE_IS_NULLPTR
    assert L.cg3mBatchPlanExecute(h.h, None, 0) == cg3m.INVALID_VALUE
    assert L.cg3mBatchPlanDestroy(None) == cg3m.INVALID_VALUE
    assert L.cg3mBatchPlanDescribe(None, None, None, None) == cg3m.INVALID_VALUE


def test_cgemm_statuses_without_device(cg3m):
    """aclblasCgemm keeps INVALID_ENUM and needs A, B whenever k > 0 (alpha == 0 included)."""
    L = cg3m.lib
    h = cg3m.Handle()
    one, zero = ctypes.byref(cg3m.cx(1)), ctypes.byref(cg3m.cx(0))
    d = ctypes.c_void_p(0x1000)
    assert L.cg3mCgemm(None, 0, 0, 2, 2, 2, one, d, 2, d, 2, zero, d, 2) == cg3m.HANDLE_IS_NULLPTR
    assert L.cg3mCgemm(h.h, 5, 0, 2, 2, 2, one, d, 2, d, 2, zero, d, 2) == cg3m.INVALID_ENUM
    assert L.aclblasCgemm(h.h, 0, 3, 2, 2, 2, one, d, 2, d, 2, zero, d, 2) == cg3m.INVALID_ENUM  # no R here
    assert L.cg3mCgemm(h.h, 0, 0, -1, 2, 2, one, d, 2, d, 2, zero, d, 2) == cg3m.INVALID_VALUE
    assert L.cg3mCgemm(h.h, 0, 0, 2, 2, 2, one, d, 1, d, 2, zero, d, 2) == cg3m.INVALID_VALUE
    assert L.cg3mCgemm(h.h, 0, 0, 2, 2, 2, None, d, 2, d, 2, zero, d, 2) == cg3m.INVALID_VALUE
    assert L.cg3mCgemm(h.h, 0, 0, 0, 2, 2, one, None, 1, None, 2, zero, None, 1) == cg3m.SUCCESS
    assert L.cg3mCgemm(h.h, 0, 0, 2, 2, 2, one, d, 2, d, 2, zero, None, 2) == cg3m.INVALID_VALUE
    # alpha == 0 still needs A and B when k > 0 (the 3m entry does not)
    assert L.cg3mCgemm(h.h, 0, 0, 2, 2, 2, zero, None, 2, d, 2, one, d, 2) == cg3m.INVALID_VALUE
    assert L.cg3mCgemm3m(h.h, 0, 0, 2, 2, 2, zero, None, 2, None, 2, one, d, 2) == cg3m.SUCCESS
    # alpha == 0, beta == 1 with valid pointers: nothing to do
    assert L.cg3mCgemm(h.h, 0, 0, 2, 2, 2, zero, d, 2, d, 2, one, d, 2) == cg3m.SUCCESS


def test_onchip_plan(cg3m):
    """The on-chip family splits K only when few tile tasks would leave SMs idle."""
    big = cg3m.plan_onchip(1024, 1024, 1024, mode=0, batch=64)
    assert big["k_partitions"] == 1 and big["tile_m"] * big["tile_n"] == 8192
    few = cg3m.plan_onchip(64, 64, 4096, mode=0, batch=1)
    assert few["k_partitions"] > 1 and few["k_span"] * (few["k_partitions"] - 1) < 4096
    # one problem: the one-launch kernel, K partitions merged in a cluster of <= 8
    assert few["path"] == 4 and few["workspace_bytes"] == 0 and few["k_partitions"] <= 8
    one4 = cg3m.plan_onchip(1024, 1024, 1024, mode=1, batch=1)
    assert (one4["tile_m"], one4["tile_n"]) != (128, 64)  # four accumulators: no 128x64 tile
    four = cg3m.plan_onchip(1024, 1024, 1024, mode=1, batch=8)
    assert four["tile_m"] * four["tile_n"] <= 4096  # no 128x64 tile with four accumulators
    # cgemm with alpha = 1, beta = 0: the FP32 planner's engine, non-finite repair in its epilogues
    big_unit = cg3m.plan_onchip(2048, 2048, 2048, mode=2, batch=1)
    assert big_unit["path"] in (2, 3) and big_unit["kernels"] >= 2  # pack, GEMM (repair in its epilogue)
    small_unit = cg3m.plan_onchip(64, 64, 64, mode=2, batch=1)
    assert small_unit["path"] == 4 and small_unit["kernels"] == 1
    with pytest.raises(cg3m.Cg3mError):
        cg3m.plan_onchip(64, 64, 64, mode=2, batch=2)


@pytest.mark.parametrize("m,n,parts,merged", [
    (512, 2048, 2, True),    # 32 pair tiles: 32 clusters of 4 CTAs fit at once (33)
    (768, 1536, 2, False),   # 36 clusters of 4 do not: pack + GEMM + merge kernel
    (512, 1408, 3, True),    # 22 clusters of 6 fit (22)
    (512, 1536, 3, False),   # 24 do not
    (768, 640, 4, True),     # 15 clusters of 8 fit (15)
    (512, 1792, 4, False),   # 28 do not
    (128, 1024, 2, False),   # one row tile: the single-CTA kernel, which writes partials
])
def test_tc_cluster_merge_gate(cg3m, m, n, parts, merged):
    """Tensor-core K splits of 2..4 merge inside the tile's cluster (pack +
    GEMM, no merge kernel) only when every cluster of 2 x parts CTAs of the
    grid is resident at once on 148 SMs; a grid that one wave holds as loose
    CTAs but not as clusters keeps the merge kernel."""
    for form in ("tf32x3", "bf16x6"):
        p = cg3m.plan("N", "N", m, n, 2048, form=form, rounding="off", k_partitions=parts)
        assert p["k_partitions"] == parts and p["path"] == 3
        assert p["kernels"] == (2 if merged else 3), (form, m, n, parts, p)
