"""C-tile sharding with the emulated call on one GPU: every rank's block, computed on its own
through the C ABI (operand offsets, leading dimensions of the full arrays), equals the same
block of the unsharded call bit for bit, for world sizes 2 to 8 and every op. The ranks run one
after another on one device; the gather over NCCL is the CPU suite's (gloo) code path."""
import pytest

pytestmark = pytest.mark.gpu


def dev_rand(torch, seed, count):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand(count, dtype=torch.float64, device="cuda", generator=g) * 2 - 1


@pytest.mark.parametrize("ta,tb,m,n,k,cplx", [("N", "N", 1000, 700, 300, False), ("T", "T", 513, 1290, 77, False),
                                              ("N", "T", 2048, 256, 1024, False), ("C", "N", 300, 500, 200, True)])
def test_blocks_equal_the_unsharded_call(oz, ta, tb, m, n, k, cplx):
    import torch
    import oz2
    from oz2 import sharded
    w = 2 if cplx else 1
    lda = (m if ta == "N" else k) + 3
    ldb = (k if tb == "N" else n) + 1
    ldc = m + 7
    A = dev_rand(torch, 1, w * lda * (k if ta == "N" else m))
    B = dev_rand(torch, 2, w * ldb * (n if tb == "N" else k))
    C0 = dev_rand(torch, 3, w * ldc * n)
    alpha, beta = (1 + 0.5j, 0.25 - 1j) if cplx else (1.5, -0.5)
    full = C0.clone()
    (oz.zgemm if cplx else oz.gemm)(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, full, ldc, 16)
    torch.cuda.synchronize()
    for world in (2, 3, 4, 8):
        sho = sharded.ShardedOzaki2(oz, world=world)
        C = C0.clone()
        for r in range(world):
            (sho.local_zgemm if cplx else sho.local_gemm)(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 16,
                                                          rank=r)
        torch.cuda.synchronize()
        oz.check_device_error()
        assert torch.equal(C.view(torch.int64), full.view(torch.int64)), world
    assert isinstance(oz, oz2.Ozaki2)
