"""The Ozaki Scheme I comparison baseline on the GPU (the reference's oz1::Ozaki1::gemm,
benchmarks/ozaki1_gpu.hpp:85-147) through the C ABI, bit for bit against the oracle's
restatement, which the CPU suite pins to the reference built for the host."""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, to_dev

pytestmark = pytest.mark.gpu


def run_oz1(oz, m, n, k, A, B, C0, L):
    import torch
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    oz.ozaki1(m, n, k, dA, A.shape[0], dB, B.shape[0], dC, C0.shape[0], L)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


def check(oracle, oz, m, n, k, A, B, L, ldc=None):
    ldc = ldc or m
    C0 = np.full((ldc, n), 7.25, order="F")
    C = run_oz1(oz, m, n, k, A, B, C0, L)
    Co = C0.copy(order="F")
    assert oracle.ozaki1(m, n, k, A, A.shape[0], B, B.shape[0], Co, ldc, L) == 0
    nd = int((bits(C) != bits(Co)).sum())
    assert nd == 0, f"{nd} entries differ from the oracle"
    assert np.all(C[m:] == 7.25)  # rows m..ldc untouched
    return C


@pytest.mark.parametrize("L", [2, 3, 5, 7, 9])
@pytest.mark.parametrize("m,n,k,kind,width", [(37, 29, 100, "u", 0), (300, 260, 1000, "wide", 12),
                                              (1, 1, 1, "int", 0), (257, 129, 4097, "u", 0)])
def test_ozaki1_against_oracle(oracle, oz, L, m, n, k, kind, width):
    A = make_mat(300 + L, m, k, m + 3, kind, width)
    B = make_mat(400 + L, k, n, k + 1, kind, width)
    check(oracle, oz, m, n, k, A, B, L, ldc=m + 5)


def test_ozaki1_accuracy_grows_with_L(oracle, oz):
    """the error against the double product falls by about 2^-7 per digit until double rounding"""
    m, n, k = 200, 150, 512
    A = make_mat(1, m, k, m, "u")
    B = make_mat(2, k, n, k, "u")
    ab = np.abs(A) @ np.abs(B)
    errs = []
    for L in range(2, 10):
        C = check(oracle, oz, m, n, k, A, B, L)
        errs.append(np.max(np.abs(C - A @ B) / ab))
    assert errs[0] > 1e-5 and errs[-1] < 1e-14
    assert all(b < a for a, b in zip(errs[:4], errs[1:5]))


def test_ozaki1_non_finite_and_zero_rows(oracle, oz):
    """an inf / NaN in a row of A or a column of B makes that row / column of C NaN; zero rows
    and columns give zeros"""
    m, n, k = 70, 50, 300
    A = make_mat(5, m, k, m, "wide", 20)
    B = make_mat(6, k, n, k, "wide", 20)
    A[3, 17] = np.inf
    A[40, 0] = np.nan
    A[10, :] = 0.0
    B[299, 7] = -np.inf
    B[:, 20] = 0.0
    C = check(oracle, oz, m, n, k, A, B, 6)
    assert np.all(np.isnan(C[3])) and np.all(np.isnan(C[40])) and np.all(np.isnan(C[:, 7]))
    fin = np.ones(m, bool)
    fin[[3, 40]] = False
    assert np.all(C[fin, 20] == 0.0) and np.all(C[10, [j for j in range(n) if j != 7]] == 0.0)


def test_ozaki1_k_chunks(oracle, oz):
    """k = 140000 needs two k chunks inside the GEMM; the int64 sums stay exact"""
    m, n, k = 40, 36, 140000
    A = make_mat(7, m, k, m, "u")
    B = make_mat(8, k, n, k, "u")
    check(oracle, oz, m, n, k, A, B, 3)


def test_ozaki1_edges_and_errors(oz):
    import torch
    A = torch.ones(64, dtype=torch.float64, device="cuda")
    B = torch.ones(64, dtype=torch.float64, device="cuda")
    C = torch.full((64,), 3.0, dtype=torch.float64, device="cuda")
    oz.ozaki1(8, 8, 0, A, 8, B, 1, C, 8, 4)  # k = 0: C = 0
    torch.cuda.synchronize()
    assert torch.count_nonzero(C).item() == 0
    C.fill_(3.0)
    oz.ozaki1(0, 8, 8, A, 1, B, 8, C, 1, 4)  # empty: nothing written
    torch.cuda.synchronize()
    assert torch.all(C == 3.0).item()
    for L in (1, 10):
        with pytest.raises(ValueError):
            oz.ozaki1(8, 8, 8, A, 8, B, 8, C, 8, L)
    with pytest.raises(ValueError):  # k 4096 = 2^31: the int32 digit products could overflow
        oz.ozaki1(1, 1, 524288, A, 1, B, 524288, C, 1, 4)
    with pytest.raises(ValueError):
        oz.ozaki1(8, 8, 8, A, 4, B, 8, C, 8, 4)  # lda < m
    assert torch.all(C == 3.0).item()
