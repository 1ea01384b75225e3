"""C-tile sharding (oz2.sharded) on CPU: the partition covers C exactly once with tile-aligned
edges, the operand offsets address op(A)'s rows and op(B)'s columns for every op, and over gloo
ranks (world sizes 2, 3 and 4, as spawned processes) the blocks plus the all-gather rebuild the
whole product on every rank. The local block is a torch product here (integer-valued inputs,
so every summation order gives the same exact result); on a GPU it is the emulated call, whose
blocks the GPU suite checks against the unsharded call bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "os2-xe_b200"))

from oz2 import sharded as sh  # noqa: E402


@pytest.mark.parametrize("world", [1, 2, 3, 4, 6, 8])
@pytest.mark.parametrize("m,n", [(1000, 300), (8192, 8192), (5, 700), (0, 40), (256, 128)])
def test_partition_covers_c_once(world, m, n):
    cover = np.zeros((m, n), np.int32)
    for r in range(world):
        (r0, r1), (c0, c1) = sh.block_of(r, world, m, n)
        assert 0 <= r0 <= r1 <= m and 0 <= c0 <= c1 <= n
        if r1 > r0 and c1 > c0:  # empty blocks (more ranks than tiles) sit at the end
            assert r0 % sh.TILE_I == 0 and c0 % sh.TILE_J == 0
            assert r1 == m or r1 % sh.TILE_I == 0
            assert c1 == n or c1 % sh.TILE_J == 0
        cover[r0:r1, c0:c1] += 1
    assert np.all(cover == 1)
    pr, pc = sh.grid_shape(world, m, n)
    assert pr * pc == world


def test_grid_prefers_square_blocks():
    assert sh.grid_shape(4, 8192, 8192) == (2, 2)
    assert sh.grid_shape(8, 8192, 8192) in ((2, 4), (4, 2))
    assert sh.grid_shape(4, 100000, 100) == (4, 1)
    assert sh.grid_shape(4, 100, 100000) == (1, 4)
    assert sh.split_range(1000, 3, 256) == [(0, 512), (512, 768), (768, 1000)]
    assert sh.split_range(100, 4, 128) == [(0, 100), (100, 100), (100, 100), (100, 100)]


def _strided(torch, X, off, rows, cols, rs, cs):
    return X.as_strided((rows, cols), (rs, cs), X.storage_offset() + off)


def torch_block(cplx, ta, tb, mb, nb, k, alpha, A, oa, lda, B, ob, ldb, beta, C, oc, ldc, s):
    """C(block) = alpha op(A)(block rows) op(B)(block columns) + beta C(block) on CPU tensors
    addressed exactly as the emulated call addresses them (offsets and leading dimensions)"""
    import torch
    if cplx:
        A, B, C = (x.view(torch.complex128) for x in (A, B, C))
    Ab = _strided(torch, A, oa, mb, k, 1, lda) if ta == "N" else _strided(torch, A, oa, mb, k, lda, 1)
    if ta == "C":
        Ab = Ab.conj()
    Bb = _strided(torch, B, ob, k, nb, 1, ldb) if tb == "N" else _strided(torch, B, ob, k, nb, ldb, 1)
    if tb == "C":
        Bb = Bb.conj()
    Cb = _strided(torch, C, oc, mb, nb, 1, ldc)
    Cb.copy_(alpha * (Ab @ Bb) + beta * Cb)


def _ints(rng, n):
    return rng.integers(-8, 9, n).astype(np.float64)


def _problem(seed, ta, tb, m, n, k, cplx):
    rng = np.random.default_rng(seed)
    lda = (m if ta == "N" else k) + 3
    ldb = (k if tb == "N" else n) + 2
    ldc = m + 5
    w = 2 if cplx else 1
    A = _ints(rng, w * lda * (k if ta == "N" else m))
    B = _ints(rng, w * ldb * (n if tb == "N" else k))
    C = _ints(rng, w * ldc * n)
    return A, lda, B, ldb, C, ldc


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


CASES = [("N", "N", 600, 300, 50, False), ("T", "N", 300, 700, 20, False), ("N", "T", 257, 129, 7, False),
         ("C", "T", 300, 260, 9, True), ("N", "N", 3, 5, 4, False)]


def _rank(rank, world, port, out):
    sys.path.insert(0, os.path.join(ROOT, "os2-xe_b200"))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from oz2 import sharded
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        res = []
        for ci, (ta, tb, m, n, k, cplx) in enumerate(CASES):
            A, lda, B, ldb, C, ldc = _problem(100 + ci, ta, tb, m, n, k, cplx)
            tA, tB, tC = (torch.from_numpy(x.copy()) for x in (A, B, C))
            want = tC.clone()
            one = sharded.ShardedOzaki2(None, compute=torch_block, world=1)
            one.compute(cplx, ta, tb, m, n, k, 1.5, tA, 0, lda, tB, 0, ldb, -0.5, want, 0, ldc, 16)
            sho = sharded.ShardedOzaki2(None, compute=torch_block)
            if rank != 0:  # inputs held by rank 0 only: the broadcast gives every rank a copy
                tA.zero_()
                tB.zero_()
            sho.broadcast(tA, tB)
            alpha, beta = (1.5 + 0j, -0.5 + 0j) if cplx else (1.5, -0.5)
            (sho.zgemm if cplx else sho.gemm)(ta, tb, m, n, k, alpha, tA, lda, tB, ldb, beta, tC, ldc, 16)
            res.append(bool(torch.equal(tC, want)))
        out.put((rank, res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_ranks_rebuild_the_product(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok in res:
        assert all(ok), (rank, ok)
