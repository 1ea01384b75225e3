"""C-tile sharding of one emulated DGEMM / ZGEMM over the ranks of a process group, one GPU per
rank: C is cut into a pr x pc grid of blocks (pr pc = world size), rank r = ri pc + ci computes
block (ri, ci) from its rows of op(A) and its columns of op(B) with the whole inner dimension,
and an optional all-gather gives every rank all of C.

Every row of op(A) and every column of op(B) is scaled on its own (the exponents come from whole
rows / columns over all k), and the CRT of an entry only sees that entry's residues, so a block
computed on its own equals the same block of the unsharded call bit for bit. No collective is
needed beyond the final gather; each rank holds A and B (a caller that holds them on one rank
broadcasts them first, `broadcast`). Block edges fall on the GEMM's output tiles (256 rows of
op(A), 128 columns of op(B)) so that no rank computes a partial tile its neighbour also pays for.

There is no counterpart in the reference (one device per Ozaki2 object); the partitioning is the
one its tiling loop (src/ozaki2_gpu.hpp:1004-1052) applies to independent (i0, j0) tiles.
"""
import math

TILE_I = 256  # output rows of op(A) per GEMM tile
TILE_J = 128  # output columns of op(B) per GEMM tile


def grid_shape(world, m, n):
    """(pr, pc) with pr pc = world whose blocks (m / pr) x (n / pc) are closest to square"""
    if world < 1:
        raise ValueError("world size must be positive")
    best = None
    for pr in range(1, world + 1):
        if world % pr:
            continue
        pc = world // pr
        bm, bn = max(m, 1) / pr, max(n, 1) / pc
        key = (abs(math.log(bm / bn)), pr)
        if best is None or key < best[0]:
            best = (key, (pr, pc))
    return best[1]


def split_range(total, parts, align):
    """`parts` consecutive [start, end) ranges covering [0, total), each a whole number of
    `align`-wide units except where the total ends; the units are spread as evenly as possible"""
    units = -(-total // align) if total > 0 else 0
    base, extra = divmod(units, parts)
    out, u = [], 0
    for p in range(parts):
        nu = base + (1 if p < extra else 0)
        out.append((min(u * align, total), min((u + nu) * align, total)))
        u += nu
    return out


def block_of(rank, world, m, n):
    """rows [r0, r1) of op(A) / C and columns [c0, c1) of op(B) / C that `rank` computes"""
    pr, pc = grid_shape(world, m, n)
    ri, ci = divmod(rank, pc)
    return split_range(m, pr, TILE_I)[ri], split_range(n, pc, TILE_J)[ci]


def operand_offsets(ta, tb, r0, c0, lda, ldb, ldc):
    """element offsets (in scalars of the operand type) of op(A) row r0, op(B) column c0 and
    C(r0, c0) in column-major storage"""
    a = r0 if ta in "Nn" else r0 * lda
    b = c0 * ldb if tb in "Nn" else c0
    return a, b, r0 + c0 * ldc


def _block_view(torch, C, ldc, r0, r1, c0, c1, cplx):
    """C(r0:r1, c0:c1) of a flat column-major array as a strided view (complex: interleaved
    pairs of doubles)"""
    if cplx:
        return C.as_strided((c1 - c0, r1 - r0, 2), (2 * ldc, 2, 1), C.storage_offset() + 2 * (r0 + c0 * ldc))
    return C.as_strided((c1 - c0, r1 - r0), (ldc, 1), C.storage_offset() + r0 + c0 * ldc)


class ShardedOzaki2:
    """`oz2.Ozaki2` calls split over the ranks of `group` (torch.distributed). `compute` replaces
    the local call (same arguments as `Ozaki2.gemm` / `zgemm` with operand offsets added) and
    exists for host-side tests of the partitioning; by default the local block runs through
    `oz` on this rank's GPU. Without a process group, `world` sets the number of blocks, so that
    one process can compute any rank's block (`local_gemm(..., rank=r)`)."""

    def __init__(self, oz, group=None, compute=None, world=None):
        import torch.distributed as dist
        self.oz = oz
        self.group = group
        self.dist = dist
        if dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, world or 1
        self.compute = compute

    def block(self, m, n, rank=None):
        return block_of(self.rank if rank is None else rank, self.world, m, n)

    def _local(self, cplx, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, rank):
        (r0, r1), (c0, c1) = block_of(rank, self.world, m, n)
        if r1 <= r0 or c1 <= c0:
            return (r0, r1), (c0, c1)
        oa, ob, oc = operand_offsets(ta, tb, r0, c0, lda, ldb, ldc)
        if self.compute is not None:
            self.compute(cplx, ta, tb, r1 - r0, c1 - c0, k, alpha, A, oa, lda, B, ob, ldb, beta, C, oc, ldc, s)
        else:
            w = 16 if cplx else 8  # bytes per scalar
            call = self.oz.zgemm if cplx else self.oz.gemm
            call(ta, tb, r1 - r0, c1 - c0, k, alpha, A.data_ptr() + w * oa, lda, B.data_ptr() + w * ob, ldb, beta,
                 C.data_ptr() + w * oc, ldc, s)
        return (r0, r1), (c0, c1)

    def local_gemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, rank=None):
        """this rank's block of C = alpha op(A) op(B) + beta C; returns its ranges"""
        return self._local(False, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s,
                           self.rank if rank is None else rank)

    def local_zgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, rank=None):
        return self._local(True, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s,
                           self.rank if rank is None else rank)

    def gather(self, C, ldc, m, n, cplx=False):
        """every rank's block into every rank's C (one all-gather of the blocks, padded to the
        largest); rows m..ldc of C stay untouched"""
        import torch
        if self.world == 1 or not self.dist.is_initialized():
            return
        w = 2 if cplx else 1
        blocks = [block_of(r, self.world, m, n) for r in range(self.world)]
        size = max((r1 - r0) * (c1 - c0) for (r0, r1), (c0, c1) in blocks) * w
        if size == 0:
            return
        mine = torch.zeros(size, dtype=C.dtype, device=C.device)
        (r0, r1), (c0, c1) = blocks[self.rank]
        cnt = (r1 - r0) * (c1 - c0) * w
        if cnt:
            mine[:cnt].copy_(_block_view(torch, C, ldc, r0, r1, c0, c1, cplx).reshape(-1))
        allb = torch.empty(self.world * size, dtype=C.dtype, device=C.device)
        self.dist.all_gather_into_tensor(allb, mine, group=self.group)
        for r, ((a0, a1), (b0, b1)) in enumerate(blocks):
            cnt = (a1 - a0) * (b1 - b0) * w
            if r == self.rank or cnt == 0:
                continue
            v = _block_view(torch, C, ldc, a0, a1, b0, b1, cplx)
            v.copy_(allb[r * size:r * size + cnt].view(v.shape))

    def gemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, gather=True):
        """C = alpha op(A) op(B) + beta C over the group: this rank's block, then (gather=True)
        all of C on every rank. A, B and C are this rank's full copies (flat float64 tensors)."""
        rng = self.local_gemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s)
        if gather:
            self.gather(C, ldc, m, n)
        return rng

    def zgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s, gather=True):
        """the complex form: A, B, C flat float64 tensors of interleaved (re, im) pairs"""
        rng = self.local_zgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s)
        if gather:
            self.gather(C, ldc, m, n, cplx=True)
        return rng

    def broadcast(self, *tensors, src=0):
        """copies of the inputs held by rank `src` onto every rank"""
        for t in tensors:
            self.dist.broadcast(t, src=src, group=self.group)
