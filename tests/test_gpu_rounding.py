"""GPU parity of the rounding-correction pass.

Reference: gemm_cgemm3m_rounding_do and its kernels (ops-blas/blas/gemm/arch35/
cgemm3m_rounding_kernel.cpp:43-497), gated at cgemm_host.cpp:234-238, and the
path-tracking fused kernel (cgemm_compute_kernel.cpp:432-474, 897-927).

FP32 form: every stage is bit-exact against the oracle -- the segmented path
GEMM (C and risk plane), the energies, the selection predicate and the
segmented prefix replay of flagged outputs -- checked on scattered output
blocks of a 2048^3 call.  The reference's SegmentCancellation known answer
(cgemm3m_test.cpp:212-240) must come back within 0.01 for every form.
"""
import numpy as np
import pytest

from gpu_util import run, sub_problem, to_dev, to_host

pytestmark = pytest.mark.gpu

N = 2048


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _square(oracle, fill, seed, scale=1.0, n=N):
    a = oracle.make_matrix(n, n, n, fill, seed)
    b = oracle.make_matrix(n, n, n, fill, seed + 1)
    if scale != 1.0:
        a = (a * np.float32(scale)).astype(np.complex64)
        b = (b * np.float32(scale)).astype(np.complex64)
    return a, b


@pytest.mark.parametrize("ops,N", [(("N", "N"), 2048), (("C", "T"), 2048), (("N", "N"), 3000), (("T", "C"), 4096),
                                   (("C", "N"), 2049)])
def test_fp32_rounding_pass_bit_exact_blocks(cg3m, oracle, cuda, h, ops, N):
    """Orders 2048, 3000 and 4096 give lane widths of 33, 47 and 65 K terms
    (ceil(n/64) | 1), replayed in chunks of 9, 12 and 17, with short or empty
    last lanes; the odd order 2049 stores the packed rows with a padded pitch."""
    import torch

    ta, tb = ops
    # Precision-form data (Im scaled by 2^e per column): about 70% of the
    # outputs are flagged, the rest keep the path GEMM's value.
    a = oracle.precision_matrix(N, N, 11)
    b = oracle.precision_matrix(N, N, 12)
    c0 = np.zeros(N * N, np.complex64)
    out, info = run(cg3m, h, torch, cuda, ta, tb, N, N, N, 1.0, a, N, b, N, 0.0, c0, N)
    assert info["rounding"] == 1 and info["kernels"] == 9
    again, _ = run(cg3m, h, torch, cuda, ta, tb, N, N, N, 1.0, a, N, b, N, 0.0, c0, N)
    assert out.tobytes() == again.tobytes()
    e = oracle.energy(N, ta, tb, a, N, b, N)
    rows = np.r_[0:8, 1000:1008, N - 8:N]
    cols = np.r_[0:6, 1500:1506, N - 6:N]
    sa, slda = sub_problem(oracle, ta, a, N, N, N, rows, 0)
    sb, sldb = sub_problem(oracle, tb, b, N, N, N, cols, 1)
    path, cpath = oracle.risk_path_rect(len(rows), len(cols), N, ta, sa, slda, tb, sb, sldb)
    P = path.reshape(len(cols), len(rows)).T
    Cm = cpath.reshape(len(cols), len(rows)).T
    flags = oracle.select_flags(P, Cm, e[rows], e[N + cols], oracle.bridge(N))
    assert flags.any() and not flags.all()
    opa = oracle.op_matrix(a, N, ta, N, N)
    opb = oracle.op_matrix(b, N, tb, N, N)
    expect = Cm.copy()
    for (r, q) in zip(*np.nonzero(flags)):
        expect[r, q] = oracle.recompute_dot(np.ascontiguousarray(opa[rows[r], :]), np.ascontiguousarray(opb[:, cols[q]]))
    got = oracle.unpack(out, N, N, N)[np.ix_(rows, cols)]
    assert got.tobytes() == expect.astype(np.complex64).tobytes()


def _mixed_density_inputs(oracle, n):
    """Uniform(-1,1) operands (nothing flagged) with five rows of op(A) and six
    adjacent columns of op(B) scaled by 1024, which flags those whole rows and
    columns through the energy term: 16 x 16 tiles crossed by one scaled row
    hold 16 flagged outputs (recomputed one by one), tiles of the six columns
    hold 96 or more (recomputed as tiles)."""
    a = oracle.make_matrix(n, n, n, "UNIFORM_1", 91)
    b = oracle.make_matrix(n, n, n, "UNIFORM_1", 92)
    rows = [5, 100, 777, 1500, n - 3]
    cols = list(range(160, 166))
    A = a.reshape(n, n)  # [col][row]: column-major n x n
    B = b.reshape(n, n)
    for r in rows:
        A[:, r] *= np.float32(1024.0)
    for c in cols:
        B[c, :] *= np.float32(1024.0)
    return a, b, rows, cols


@pytest.mark.parametrize("form", ["fp32", "bf16x6"])
def test_rounding_pass_sparse_and_dense_tiles(cg3m, oracle, cuda, h, form):
    """Tiles with few flagged outputs go to the per-output kernel, dense ones
    to the tile kernel; each flagged output is recomputed exactly once.  FP32:
    every checked block is bit-exact against the oracle (path GEMM value where
    unflagged, segmented replay where flagged); FP64 recompute: flagged
    outputs within one FP32 rounding of the FP64 product."""
    import torch

    n = 2048
    a, b, srows, scols = _mixed_density_inputs(oracle, n)
    c0 = np.zeros(n * n, np.complex64)
    out, info = run(cg3m, h, torch, cuda, "N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c0, n, form=form)
    assert info["rounding"] == 1
    st = h.rounding_stats()
    assert st["dense_outputs"] > 0 and st["sparse_outputs"] > 0
    assert st["dense_outputs"] + st["sparse_outputs"] == st["flagged"]
    if form != "fp32":
        assert st["exact_tiles"] > 0 and st["fallback_outputs"] <= st["dense_outputs"]
    e = oracle.energy(n, "N", "N", a, n, b, n)
    rows = np.r_[0:8, 96:104, 770:780, n - 8:n]
    cols = np.r_[0:6, 156:170, 1500:1506, n - 6:n]
    sa, slda = sub_problem(oracle, "N", a, n, n, n, rows, 0)
    sb, sldb = sub_problem(oracle, "N", b, n, n, n, cols, 1)
    opa = oracle.op_matrix(a, n, "N", n, n)
    opb = oracle.op_matrix(b, n, "N", n, n)
    got = oracle.unpack(out, n, n, n)[np.ix_(rows, cols)]
    if form == "fp32":
        path, cpath = oracle.risk_path_rect(len(rows), len(cols), n, "N", sa, slda, "N", sb, sldb)
        P = path.reshape(len(cols), len(rows)).T
        Cm = cpath.reshape(len(cols), len(rows)).T
        flags = oracle.select_flags(P, Cm, e[rows], e[n + cols], oracle.bridge(n))
        assert flags.any() and not flags.all()
        expect = Cm.copy()
        for (r, q) in zip(*np.nonzero(flags)):
            expect[r, q] = oracle.recompute_dot(np.ascontiguousarray(opa[rows[r], :]),
                                                np.ascontiguousarray(opb[:, cols[q]]))
        assert got.tobytes() == expect.astype(np.complex64).tobytes()
    else:
        z = opa[rows, :].astype(np.complex128) @ opb[:, cols].astype(np.complex128)
        for r in range(len(rows)):
            for q in range(len(cols)):
                if rows[r] in srows or cols[q] in scols:  # flagged through the energy term
                    x = complex(got[r, q])
                    assert abs(x.real - z[r, q].real) <= np.spacing(np.float32(abs(z[r, q].real)))
                    assert abs(x.imag - z[r, q].imag) <= np.spacing(np.float32(abs(z[r, q].imag)))


def _kat_inputs(residual):
    size, tps = 2048, 33
    a = np.zeros(size * size, np.complex64)
    b = np.zeros(size * size, np.complex64)
    for inner in range(40 * tps):
        a[inner * size] = 1.0  # A(0, inner)
        b[inner] = 4096.1 if inner < 20 * tps else -4096.1  # B(inner, 0)
    a[(size - 1) * size] = 1.0
    b[size - 1] = residual
    return a, b


@pytest.mark.parametrize("form", ["fp32", "tf32x3", "bf16x6", "bf16x9"])
def test_segment_cancellation_kat(cg3m, oracle, cuda, h, form):
    """cgemm3m_test.cpp:212-240: C(0,0) = residual within 0.01 (sequential FP32
    accumulation alone drifts by ~0.015); everything else is exactly zero."""
    import torch

    size = 2048
    for residual in (0.0, 1.0):
        a, b = _kat_inputs(residual)
        c0 = np.zeros(size * size, np.complex64)
        out, info = run(cg3m, h, torch, cuda, "N", "N", size, size, size, 1.0, a, size, b, size, 0.0, c0, size,
                        form=form)
        assert info["rounding"] == 1
        assert abs(out[0].real - residual) <= 0.01 and abs(out[0].imag) <= 0.01, out[0]
        expect = c0.copy()
        expect[0] = residual
        assert oracle.verify_cgemm3m(out, expect, c0, size, size, size)[0]


@pytest.mark.parametrize("form", ["tf32x3", "bf16x6", "bf16x9"])
def test_tc_rounding_pass_recomputes_in_fp64(cg3m, oracle, cuda, h, form):
    """Tensor-core forms recompute flagged outputs in FP64: those outputs are
    within one FP32 rounding of the FP64 product, and the whole result's
    normwise error is no worse than with the pass off."""
    import torch

    a = oracle.precision_matrix(N, N, 21)
    b = oracle.precision_matrix(N, N, 22)
    A, B = to_dev(a, torch, cuda), to_dev(b, torch, cuda)
    C = torch.zeros(N * N, dtype=torch.complex64, device=cuda)
    ref = torch.empty(N * N, dtype=torch.complex128, device=cuda)
    h.zgemm_reference("N", "N", N, N, N, 1.0, A, N, B, N, 0.0, C, N, ref)
    info = h.cgemm3m("N", "N", N, N, N, 1.0, A, N, B, N, 0.0, C, N, form=form)
    assert info["rounding"] == 1
    on = h.error_report(N, N, C, N, ref)
    st = h.rounding_stats()
    # every 256 x 256 tile is dense on this data: int8 slice products, few fallbacks
    assert st["exact_tiles"] == (N // 256) ** 2 and st["sparse_outputs"] == 0
    assert st["fallback_outputs"] < 0.05 * st["flagged"]
    got_on = C.clone()
    h.cgemm3m("N", "N", N, N, N, 1.0, A, N, B, N, 0.0, C, N, form=form, rounding="off")
    off = h.error_report(N, N, C, N, ref)
    torch.cuda.synchronize()
    assert on["normwise"] <= off["normwise"]
    changed = (got_on != C).cpu().numpy()
    assert changed.any()
    x = got_on.cpu().numpy()[changed].astype(np.complex128)
    z = ref.cpu().numpy()[changed]
    assert np.all(np.abs(x.real - z.real) <= np.spacing(np.abs(z.real).astype(np.float32)))
    assert np.all(np.abs(x.imag - z.imag) <= np.spacing(np.abs(z.imag).astype(np.float32)))




@pytest.mark.parametrize("form", ["tf32x3", "bf16x6"])
def test_tc_pass_tiles_taken_and_form_products(cg3m, oracle, cuda, h, form):
    """Tensor-core forms: every output of a 256 x 256 tile the exact recompute
    takes is within one FP32 rounding of the FP64 product, flagged or not;
    outside those tiles the unflagged outputs are the form's own products byte
    for byte (the same call with the pass off) and the flagged ones (the
    scaled rows, recomputed one by one in FP64) are within one FP32 rounding."""
    import torch

    n = 2048
    a, b, srows, scols = _mixed_density_inputs(oracle, n)
    c0 = np.zeros(n * n, np.complex64)
    on, info = run(cg3m, h, torch, cuda, "N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c0, n, form=form)
    assert info["rounding"] == 1
    st = h.rounding_stats()
    # the six scaled columns 160..165 make every 16 x 16 tile of columns 160..175 dense,
    # so the exact recompute takes the 256-column strip 0..255 in every row band
    assert st["exact_tiles"] == n // 256 and st["exact_positions"] == n * 256
    # the pass's form products run unsplit over K: the comparison call too
    off, _ = run(cg3m, h, torch, cuda, "N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c0, n, form=form,
                 rounding="off", k_partitions=1)
    On = oracle.unpack(on, n, n, n)
    Off = oracle.unpack(off, n, n, n)
    opa = oracle.op_matrix(a, n, "N", n, n).astype(np.complex128)
    opb = oracle.op_matrix(b, n, "N", n, n).astype(np.complex128)

    def within_one_rounding(x, z):
        x = x.astype(np.complex128)
        sr = np.spacing(np.abs(z.real).astype(np.float32)).astype(np.float64)
        si = np.spacing(np.abs(z.imag).astype(np.float32)).astype(np.float64)
        return np.all(np.abs(x.real - z.real) <= sr) and np.all(np.abs(x.imag - z.imag) <= si)

    # taken strip: sampled rows (scaled and plain), all 256 columns
    rows = np.r_[0:8, srows, 1000:1008, n - 8:n]
    z = opa[rows, :] @ opb[:, 0:256]
    assert within_one_rounding(On[rows, 0:256], z)
    # outside it: plain rows keep the form's products exactly, scaled rows are recomputed
    plain = np.setdiff1d(np.arange(n), srows)
    assert On[np.ix_(plain, np.arange(256, n))].tobytes() == Off[np.ix_(plain, np.arange(256, n))].tobytes()
    z = opa[srows, :] @ opb[:, 256:]
    assert within_one_rounding(On[srows, 256:], z)


@pytest.mark.parametrize("form", ["tf32x3", "bf16x6"])
def test_tc_pass_row_band_taken(cg3m, oracle, cuda, h, form):
    """The transposed layout: six adjacent op(A) rows scaled by 1024 make every
    tile of the first 256-row band dense, so the exact recompute takes that
    band across all columns and the rest of the form's planes is packed for
    the other op(A) row bands only.  Outside the band the unflagged outputs are
    the form's own products byte for byte and the scaled columns' outputs are
    within one FP32 rounding; inside it every output is within one rounding."""
    import torch

    n = 2048
    a = oracle.make_matrix(n, n, n, "UNIFORM_1", 93)
    b = oracle.make_matrix(n, n, n, "UNIFORM_1", 94)
    srows = list(range(160, 166))
    scols = [7, 300, 1201, n - 2]
    A = a.reshape(n, n)  # [col][row]
    B = b.reshape(n, n)
    for r in srows:
        A[:, r] *= np.float32(1024.0)
    for c in scols:
        B[c, :] *= np.float32(1024.0)
    c0 = np.zeros(n * n, np.complex64)
    on, info = run(cg3m, h, torch, cuda, "N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c0, n, form=form)
    assert info["rounding"] == 1
    st = h.rounding_stats()
    assert st["exact_tiles"] == n // 256 and st["exact_positions"] == 256 * n
    off, _ = run(cg3m, h, torch, cuda, "N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c0, n, form=form,
                 rounding="off", k_partitions=1)
    On = oracle.unpack(on, n, n, n)
    Off = oracle.unpack(off, n, n, n)
    opa = oracle.op_matrix(a, n, "N", n, n).astype(np.complex128)
    opb = oracle.op_matrix(b, n, "N", n, n).astype(np.complex128)

    def within_one_rounding(x, z):
        x = x.astype(np.complex128)
        sr = np.spacing(np.abs(z.real).astype(np.float32)).astype(np.float64)
        si = np.spacing(np.abs(z.imag).astype(np.float32)).astype(np.float64)
        return np.all(np.abs(x.real - z.real) <= sr) and np.all(np.abs(x.imag - z.imag) <= si)

    # taken band: all 256 rows, sampled columns (scaled and plain)
    cols = np.r_[0:8, scols, 1000:1008, n - 8:n]
    assert within_one_rounding(On[0:256][:, cols], opa[0:256, :] @ opb[:, cols])
    # outside it: plain columns keep the form's products exactly, scaled columns are recomputed
    plain = np.setdiff1d(np.arange(n), scols)
    assert On[np.ix_(np.arange(256, n), plain)].tobytes() == Off[np.ix_(np.arange(256, n), plain)].tobytes()
    assert within_one_rounding(On[256:, :][:, scols], opa[256:, :] @ opb[:, scols])


@pytest.mark.parametrize("form", ["tf32x3", "bf16x6"])
def test_tc_pass_odd_order_edges(cg3m, oracle, cuda, h, form):
    """Order 2077 (a rounding-gated size of the reference's performance table,
    not a multiple of the 256 x 256 exact tile): the last row and column of
    tiles are partial, the residue planes padded.  Precision-form data flags
    every tile, so every output, edges included, is within one FP32 rounding
    of the FP64 product."""
    import torch

    n = 2077
    a = oracle.precision_matrix(n, n, 41)
    b = oracle.precision_matrix(n, n, 42)
    c0 = np.zeros(n * n, np.complex64)
    out, info = run(cg3m, h, torch, cuda, "N", "N", n, n, n, 1.0, a, n, b, n, 0.0, c0, n, form=form)
    assert info["rounding"] == 1
    st = h.rounding_stats()
    tiles = (n + 255) // 256
    assert st["exact_tiles"] == tiles * tiles and st["exact_positions"] == n * n
    got = oracle.unpack(out, n, n, n)
    opa = oracle.op_matrix(a, n, "N", n, n).astype(np.complex128)
    opb = oracle.op_matrix(b, n, "N", n, n).astype(np.complex128)
    rows = np.r_[0:8, 2040:2077]   # the partial last row band and the rows before it
    cols = np.r_[0:16, 2040:2077]
    z = opa[rows, :] @ opb[:, cols]
    x = got[np.ix_(rows, cols)].astype(np.complex128)
    ur = np.spacing(np.abs(z.real).astype(np.float32)).astype(np.float64)
    ui = np.spacing(np.abs(z.imag).astype(np.float32)).astype(np.float64)
    assert np.all(np.abs(x.real - z.real) <= ur) and np.all(np.abs(x.imag - z.imag) <= ui)
