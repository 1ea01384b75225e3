"""The Ozaki Scheme I comparison baseline: the oracle's restatement against the reference's own
oz1::Ozaki1 (built for the host), bit for bit."""
import numpy as np
import pytest

from common import bits, make_mat


@pytest.mark.parametrize("L", [2, 4, 6, 9])
@pytest.mark.parametrize("m,n,k,kind,width", [(37, 29, 100, "u", 0), (64, 48, 257, "wide", 12), (5, 7, 1, "int", 0)])
def test_ozaki1_oracle_equals_reference(oracle, ref, L, m, n, k, kind, width):
    A = make_mat(900 + L, m, k, m + 2, kind, width)
    B = make_mat(950 + L, k, n, k + 1, kind, width)
    Co = np.zeros((m, n), order="F")
    Cr = np.zeros((m, n), order="F")
    assert oracle.ozaki1(m, n, k, A, m + 2, B, k + 1, Co, m, L) == 0
    assert ref.ozaki1(m, n, k, A, m + 2, B, k + 1, Cr, m, L) == 0
    assert np.array_equal(bits(Co), bits(Cr))


def test_ozaki1_errors_and_accuracy(oracle):
    A = make_mat(1, 50, 60, 50, "u")
    B = make_mat(2, 60, 40, 60, "u")
    C = np.zeros((50, 40), order="F")
    assert oracle.ozaki1(50, 40, 60, A, 50, B, 60, C, 50, 1) != 0
    assert oracle.ozaki1(50, 40, 600000, A, 50, B, 60, C, 50, 4) != 0
    assert oracle.ozaki1(50, 40, 60, A, 50, B, 60, C, 50, 8) == 0
    # 7 L - 2 = 54 bits per element: close to a double product
    ref = A @ B
    assert np.max(np.abs(C - ref) / (np.abs(A) @ np.abs(B))) < 1e-14
