"""Multi-process (gloo, world size 2, CPU) tests of the N > 1 host logic:
column sharding of the output, the block offsets each rank passes to the
library, and the max-over-ranks timing that bench.py uses under torchrun."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import sys

    sys.path[:0] = [os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                 "ascend-open-source-contributions_b200"),
                    os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")]
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from cg3m import dist as cdist
    import oracle as O

    # max over ranks
    got = cdist.max_over_ranks(1.5 + rank)
    # each rank computes its column block with the oracle's model; rank 0 gathers
    m, n, k = 9, 11, 7
    a = O.make_matrix(m, k, m, "UNIFORM_1", 3)
    b = O.make_matrix(n, k, n + 2, "UNIFORM_1", 4)   # op(B) = T: stored n x k
    c = np.zeros(m * n, np.complex64)
    first, cols = cdist.shard_columns(n, world, rank)
    b_off, c_off = cdist.column_block_offsets("T", n + 2, m, first)
    block = c[c_off:c_off + m * cols].copy()
    O.cgemm3m_fp32_model("N", "T", m, cols, k, 1.0, a, m, b[b_off:], n + 2, 0.0, block, m)
    import torch

    t = torch.from_numpy(np.ascontiguousarray(block.view(np.float32)))
    parts = [None] * world
    dist.all_gather_object(parts, (first, cols, t.numpy()))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        full = np.zeros(m * n, np.complex64)
        for f, cnt, arr in parts:
            full[f * m:(f + cnt) * m] = arr.view(np.complex64)
        whole = np.zeros(m * n, np.complex64)
        O.cgemm3m_fp32_model("N", "T", m, n, k, 1.0, a, m, b, n + 2, 0.0, whole, m)
        q.put((got, full.tobytes() == whole.tobytes()))
    else:
        q.put((got, True))


def test_two_rank_sharding_and_timing():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[0] == 2.5 for r in results)
    assert all(r[1] for r in results)


@pytest.mark.parametrize("n,world", [(4096, 8), (1000, 3), (5, 8), (1, 2)])
def test_shard_columns_cover_exactly_once(n, world):
    import sys

    from cg3m import dist as cdist

    seen = []
    for r in range(world):
        first, cols = cdist.shard_columns(n, world, r)
        seen.extend(range(first, first + cols))
    assert seen == list(range(n))
