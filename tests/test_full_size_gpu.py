"""The configurations of the benchmark table at their full sizes, checked through properties that
do not depend on size: a block of C (full k) equals the oracle's result for that block bit for
bit (row and column scalings use whole rows and columns, so a block is computed exactly as in
the full product), the op pairs agree bit for bit with the NN product of explicitly transposed
inputs, and a tiled run under a workspace limit equals the untiled one."""
import numpy as np
import pytest

from common import bits

pytestmark = pytest.mark.gpu

BLK = 192


def dev_uniform(torch, seed, count):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand(count, dtype=torch.float64, device="cuda", generator=g) * 2 - 1


def dev_phi(torch, seed, count, phi):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u = torch.rand(count, dtype=torch.float64, device="cuda", generator=g) - 0.5
    return u * torch.exp(phi * torch.randn(count, dtype=torch.float64, device="cuda", generator=g))


def col_major_block(t, ld, ncols, r0, r1, c0, c1):
    """rows r0:r1, columns c0:c1 of a column-major (ld x ncols) device array, as a Fortran numpy array"""
    return np.asfortranarray(t.view(ncols, ld)[c0:c1, r0:r1].cpu().numpy().T)


def check_block(oracle, torch, m, n, k, alpha, A, B, beta, C0, C, ldc, s, i0=0, j0=0, b=BLK):
    """C[i0:i0+b, j0:j0+b] against the oracle on A's rows and B's columns (NN, lda = m, ldb = k)"""
    Ab = col_major_block(A, m, k, i0, i0 + b, 0, k)
    Bb = col_major_block(B, k, n, 0, k, j0, j0 + b)
    Cb = col_major_block(C0, ldc, n, i0, i0 + b, j0, j0 + b)
    assert oracle.dgemm("N", "N", b, b, k, alpha, Ab, b, Bb, k, beta, Cb, b, s) == 0
    got = col_major_block(C, ldc, n, i0, i0 + b, j0, j0 + b)
    assert np.array_equal(bits(got), bits(Cb))


@pytest.mark.parametrize("s", [8, 12, 16])
def test_c2_dgemm_8192_blocks_and_op_pairs(oracle, oz, s):
    """DGEMM 8192^3, alpha 1.5, beta -0.5, ldc = m + 16, U[-1,1): two blocks against the oracle;
    NT, TN, TT with transposed copies equal NN bit for bit"""
    import torch
    m = n = k = 8192
    ldc = m + 16
    A = dev_uniform(torch, 11, m * k)
    B = dev_uniform(torch, 12, k * n)
    C0 = dev_uniform(torch, 13, ldc * n)
    C = C0.clone()
    oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, s)
    torch.cuda.synchronize()
    check_block(oracle, torch, m, n, k, 1.5, A, B, -0.5, C0, C, ldc, s)
    check_block(oracle, torch, m, n, k, 1.5, A, B, -0.5, C0, C, ldc, s, i0=m - BLK, j0=4096)
    At = A.view(k, m).t().contiguous().view(-1)  # op(At) = A with At stored k x m
    Bt = B.view(n, k).t().contiguous().view(-1)
    for ta, tb, AA, lda, BB, ldb in (("N", "T", A, m, Bt, n), ("T", "N", At, k, B, k), ("T", "T", At, k, Bt, n)):
        C2 = C0.clone()
        oz.gemm(ta, tb, m, n, k, 1.5, AA, lda, BB, ldb, -0.5, C2, ldc, s)
        torch.cuda.synchronize()
        assert torch.equal(C2.view(torch.int64), C.view(torch.int64)), (ta, tb)


@pytest.mark.parametrize("phi,s", [(1.0, 20), (4.0, 24)])
def test_c2_phi_set_8192(oracle, oz, phi, s):
    """DGEMM 8192^3 with (u - 0.5) exp(phi g) inputs at s = 20 and 24 (wide limb path)"""
    import torch
    m = n = k = 8192
    ldc = m + 16
    A = dev_phi(torch, 21, m * k, phi)
    B = dev_phi(torch, 22, k * n, phi)
    C0 = dev_uniform(torch, 23, ldc * n)
    C = C0.clone()
    oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, s)
    torch.cuda.synchronize()
    check_block(oracle, torch, m, n, k, 1.5, A, B, -0.5, C0, C, ldc, s, i0=1000, j0=7000)


def test_c2_k_split_262144(oracle, oz):
    """m = n = 1024, k = 262144 (k chunks inside the GEMM), s = 16"""
    import torch
    m = n = 1024
    k = 262144
    A = dev_uniform(torch, 31, m * k)
    B = dev_uniform(torch, 32, k * n)
    C0 = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    C = C0.clone()
    oz.gemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, 16)
    torch.cuda.synchronize()
    assert oz.last_tiling().k_chunks == 3
    check_block(oracle, torch, m, n, k, 1.0, A, B, 0.0, C0, C, m, 16, i0=512, j0=256, b=64)


def zblock(t, ld, ncols, r0, r1, c0, c1):
    """complex block of an interleaved column-major (ld x ncols) complex array"""
    v = t.view(ncols, ld, 2)[c0:c1, r0:r1].cpu().numpy()
    return np.asfortranarray((v[..., 0] + 1j * v[..., 1]).T)


def test_c3_zgemm_4096_conj(oracle, oz):
    """ZGEMM 4096^3, op(A) = C, op(B) = N, alpha (1, 0.5), beta (0.25, -1), ldc = m + 8, s = 16"""
    import torch
    m = n = k = 4096
    ldc = m + 8
    A = dev_uniform(torch, 41, 2 * k * m)  # op(A) = A^H: A stored k x m
    B = dev_uniform(torch, 42, 2 * k * n)
    C0 = dev_uniform(torch, 43, 2 * ldc * n)
    C = C0.clone()
    oz.zgemm("C", "N", m, n, k, 1 + 0.5j, A, k, B, k, 0.25 - 1j, C, ldc, 16)
    torch.cuda.synchronize()
    b, i0, j0 = 128, 2048, 100
    Ab = zblock(A, k, m, 0, k, i0, i0 + b)  # k x b: columns i0.. of the stored A
    Bb = zblock(B, k, n, 0, k, j0, j0 + b)
    Cb = zblock(C0, ldc, n, i0, i0 + b, j0, j0 + b)
    assert oracle.zgemm("C", "N", b, b, k, 1 + 0.5j, Ab, k, Bb, k, 0.25 - 1j, Cb, b, 16) == 0
    got = zblock(C, ldc, n, i0, i0 + b, j0, j0 + b)
    assert np.array_equal(bits(got), bits(Cb))


def test_c3_zgemm_non_square_under_4gb(oracle, oz):
    """ZGEMM 3000 x 5000 x 2000 under a 4 GB workspace limit (which the 1-byte residues fit
    untiled) and under 512 MB (tiled): both equal the unlimited run bit for bit, and a block
    equals the oracle"""
    import torch
    import oz2
    m, n, k = 3000, 5000, 2000
    A = dev_uniform(torch, 51, 2 * m * k)
    B = dev_uniform(torch, 52, 2 * k * n)
    C0 = dev_uniform(torch, 53, 2 * m * n)
    C = C0.clone()
    oz.set_workspace_limit(0)
    oz.zgemm("N", "N", m, n, k, 1 + 0.5j, A, m, B, k, 0.25 - 1j, C, m, 16)
    torch.cuda.synchronize()
    for limit, tiled in ((4 << 30, False), (512 << 20, True)):
        lim = oz2.Ozaki2(torch.cuda.current_stream())
        try:
            lim.set_workspace_limit(limit)
            C2 = C0.clone()
            lim.zgemm("N", "N", m, n, k, 1 + 0.5j, A, m, B, k, 0.25 - 1j, C2, m, 16)
            torch.cuda.synchronize()
            t = lim.last_tiling()
            assert t.workspace_bytes <= limit and (t.pm * t.pn > 1) == tiled, (limit, t)
        finally:
            lim.close()
        assert torch.equal(C2.view(torch.int64), C.view(torch.int64))
    b, i0, j0 = 96, 2900, 4000
    Ab = zblock(A, m, k, i0, i0 + b, 0, k)
    Bb = zblock(B, k, n, 0, k, j0, j0 + b)
    Cb = zblock(C0, m, n, i0, i0 + b, j0, j0 + b)
    assert oracle.zgemm("N", "N", b, b, k, 1 + 0.5j, Ab, b, Bb, k, 0.25 - 1j, Cb, b, 16) == 0
    assert np.array_equal(bits(zblock(C, m, n, i0, i0 + b, j0, j0 + b)), bits(Cb))


def test_c1_dgemm_1024_full_against_oracle(oracle, oz):
    """DGEMM 1024^3 NN, alpha 1, beta 0, U[-1,1), s = 16: every entry against the oracle"""
    import torch
    m = n = k = 1024
    A = dev_uniform(torch, 61, m * k)
    B = dev_uniform(torch, 62, k * n)
    C = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    oz.gemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, 16)
    torch.cuda.synchronize()
    check_block(oracle, torch, m, n, k, 1.0, A, B, 0.0, C.clone().zero_(), C, m, 16, b=1024)
