"""GPU parity of the one-launch FP32 engine (engine 2 of cg3mCgemm3mEx): one
kernel that reads the caller's interleaved matrices and merges its K
partitions inside a thread-block cluster.

1. Every tile shape x partition count (1..8) is bit-identical to the oracle's
   model of the plain FP32 3M arithmetic with the reported K span, on ragged
   shapes with padded leading dimensions (padding bytes untouched), every op
   kind (R included) and general alpha/beta.
2. For the same K split the one-launch engine and the packed engine (pack
   kernel + TMA-fed GEMM + merge kernel) give the same bytes, non-finite
   inputs included.
3. The planner's own choice for small problems is bit-exact against the model.
"""
import numpy as np
import pytest

from gpu_util import run, same_bits

pytestmark = pytest.mark.gpu

OPS4 = ["N", "T", "C", "R"]


@pytest.fixture(scope="module")
def h(cg3m, cuda):
    return cg3m.Handle()


def _operands(oracle, ta, tb, m, n, k, pad, fill, seed):
    ar, ac = oracle.stored_shape(ta, m, k)
    br, bc = oracle.stored_shape(tb, k, n)
    lda, ldb, ldc = ar + pad, br + pad, m + pad
    a = oracle.make_matrix(ar, ac, lda, fill, seed)
    b = oracle.make_matrix(br, bc, ldb, fill, seed + 1)
    c = oracle.make_matrix(m, n, ldc, fill, seed + 2)
    return a, lda, b, ldb, c, ldc


@pytest.mark.parametrize("tile", [1, 2, 3, 4, 5, 6])
def test_every_tile_and_split_matches_model(cg3m, oracle, cuda, h, tile):
    import torch

    rng = np.random.default_rng(4100 + tile)
    for parts in range(1, 9):
        ta, tb = OPS4[int(rng.integers(4))], OPS4[int(rng.integers(4))]
        m, n, k = int(rng.integers(1, 200)), int(rng.integers(1, 200)), int(rng.integers(130, 700))
        alpha, beta = complex(0.75, -0.5), complex(0.5, 0.25) if parts % 2 else complex(0, 0)
        a, lda, b, ldb, c, ldc = _operands(oracle, ta, tb, m, n, k, 3, "RANDOM_NORM_5_5", 900 + 10 * tile + parts)
        out, info = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                        engine="onchip", onchip_tile=tile, k_partitions=parts)
        assert info["path"] == 4 and info["kernels"] == 1 and info["workspace_bytes"] == 0
        assert (info["tile_m"], info["tile_n"]) == cg3m.ONCHIP_TILES[tile - 1]
        assert 1 <= info["k_partitions"] <= parts
        model = c.copy()
        oracle.cgemm3m_fp32_model(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
        assert same_bits(out, model), (tile, parts, ta, tb, m, n, k, info)
        # rows past m in every column are padding: untouched
        assert out.reshape(n, ldc)[:, m:].tobytes() == c.reshape(n, ldc)[:, m:].tobytes()


@pytest.mark.parametrize("fill", ["RANDOM_NORM_5_5", "RANDOM_EXTREME", "VALUE_NORM_INF", "VALUE_NORM_NAN"])
def test_same_bits_as_packed_engine(cg3m, oracle, cuda, h, fill):
    import torch

    shapes = [("N", "N", 128, 128, 128), ("T", "C", 257, 65, 1000), ("C", "N", 19, 300, 1174),
              ("N", "T", 464, 21, 1663), ("T", "N", 33, 33, 17)]
    for s, (ta, tb, m, n, k) in enumerate(shapes):
        alpha, beta = complex(1.25, 0.5), complex(-0.5, 0.75)
        a, lda, b, ldb, c, ldc = _operands(oracle, ta, tb, m, n, k, 5, fill, 5100 + 7 * s)
        one, info = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                        rounding="off", engine="onchip")
        packed, pinfo = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                            rounding="off", engine="packed", k_partitions=info["k_partitions"])
        assert pinfo["k_span"] == info["k_span"]
        assert same_bits(one, packed), (fill, ta, tb, m, n, k, info)


def test_planner_choice_small_shapes(cg3m, oracle, cuda, h):
    import torch

    shapes = [("N", "N", 128, 128, 128), ("N", "N", 256, 256, 256), ("T", "N", 19, 1686, 1174),
              ("C", "C", 56, 190, 1858), ("N", "T", 464, 21, 1663), ("N", "N", 32, 808, 184),
              ("T", "N", 424, 1322, 40)]
    for s, (ta, tb, m, n, k) in enumerate(shapes):
        alpha, beta = complex(1, 0), complex(0, 0)
        a, lda, b, ldb, c, ldc = _operands(oracle, ta, tb, m, n, k, 0, "RANDOM_NORM_5_5", 5300 + 7 * s)
        out, info = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
        again, _ = run(cg3m, h, torch, cuda, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
        assert out.tobytes() == again.tobytes()
        model = c.copy()
        oracle.cgemm3m_fp32_model(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, model, ldc, span=info["k_span"])
        assert same_bits(out, model), (ta, tb, m, n, k, info)
