"""The certified number of moduli on CPU: the entrywise a-priori bound the library's certificate
evaluates (restated in numpy with the exact-enough FP64 |A||B|) is checked against the oracle's
emulation itself. At the certified s every entry of the oracle's product meets the DGEMM-level
target |C - AB| <= k 2^-53 (|A||B|)_ij against a double-double product, on inputs whose rows
span up to 2^90 (where the largest-gap analytic rule sends the tile to native FP64), and the
certified s is never above the analytic s."""
import numpy as np
import pytest

import adaptive_oracle as ao
from common import bits  # noqa: F401  (shared fixtures module)


def heavy(seed, rows, cols, phi, offsets, axis):
    rng = np.random.default_rng(seed)
    X = (rng.random((rows, cols)) - 0.5) * np.exp(phi * rng.standard_normal((rows, cols)))
    shape = (rows, 1) if axis == 0 else (1, cols)
    return np.asfortranarray(X * np.ldexp(1.0, rng.integers(-offsets, offsets + 1, shape)))


@pytest.mark.parametrize("n,k,phi,offsets", [(96, 150, 0.0, 0), (120, 300, 2.0, 20), (80, 500, 4.0, 40),
                                             (64, 700, 6.0, 40), (100, 90, 8.0, 40), (70, 1000, 1.0, 0)])
def test_certified_s_meets_the_target(oracle, n, k, phi, offsets):
    A = heavy(1000 + n, n, k, phi, offsets, 0)
    B = heavy(2000 + n, k, n, phi, offsets, 1)
    s = ao.certified_s(oracle, A, B)
    feats, s_an = ao.tile_features(oracle, [("N", "N", n, n, k, A, B)])
    assert s <= int(s_an[0])
    if s > 24:
        return
    C = np.zeros((n, n), order="F")
    assert oracle.dgemm("N", "N", n, n, k, 1.0, A, n, B, k, 0.0, C, n, s) == 0
    hi, lo = oracle.dd_gemm("N", "N", n, n, k, A, n, B, k)
    hi = np.asarray(hi).reshape((n, n), order="F")
    lo = np.asarray(lo).reshape((n, n), order="F")
    err = np.abs((C - hi) - lo)
    tgt = k * 2.0 ** -53 * (np.abs(A) @ np.abs(B))
    assert np.all(err <= tgt), (s, float(np.max(err / np.where(tgt > 0, tgt, 1))))


def test_certified_s_edges(oracle):
    A = heavy(5, 40, 64, 1.0, 0, 0)
    B = heavy(6, 64, 30, 1.0, 0, 1)
    Z = np.zeros_like(A)
    assert ao.certified_s(oracle, Z, B) == 2  # every entry exact
    A2 = A.copy()
    A2[3, 5] = np.inf
    assert ao.certified_s(oracle, A2, B) == ao.NATIVE
    assert ao.certified_s(oracle, A[:, :2], B[:2, :]) == ao.NATIVE  # k < 3
