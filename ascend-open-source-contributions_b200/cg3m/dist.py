"""Multi-GPU use of cgemm3m: output-column sharding and max-over-ranks timing.

The product shards with no exchange: C(:, j) needs all of op(A) and only
column j of op(B), so rank r of G owns a contiguous block of columns and
multiplies op(A) by its own block of op(B) (no collective is needed on the
data path).  Timing across ranks takes the maximum
of the per-rank device times.
"""
from __future__ import annotations


def shard_columns(n: int, world: int, rank: int):
    """(first column, number of columns) of rank's block; blocks are contiguous,
    cover [0, n) exactly once, and differ in size by at most one column."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(n, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def column_block_offsets(transb: str, ldb: int, ldc: int, first: int):
    """Element offsets of a column block's first column in B (op(B) columns are
    stored columns for N/R, stored rows for T/C) and in C."""
    b_off = first * ldb if transb in ("N", "R") else first
    return b_off, first * ldc


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the default process group (identity when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cgemm3m_local_block(handle, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, world, rank, **kw):
    """Runs this rank's column block of C <- alpha*op(A)*op(B) + beta*C on flat
    complex64 device tensors holding the full A, B, C (each rank touches only
    its own columns of B and C)."""
    first, cols = shard_columns(n, world, rank)
    if cols == 0:
        return None
    b_off, c_off = column_block_offsets(transb, ldb, ldc, first)
    return handle.cgemm3m(transa, transb, m, cols, k, alpha, A, lda, B[b_off:], ldb, beta, C[c_off:], ldc, **kw)
