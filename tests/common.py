"""Shared helpers of the test suite: exact seeded inputs, oracle access, device round trips.

Inputs come from a counter-based splitmix64 stream turned into doubles with integer operations
and exact power-of-two scalings only, so the same seed gives bit-identical matrices on every
machine and numpy version (golden fixtures store outputs only).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "os2-xe_b200"))
GOLDEN = os.path.join(ROOT, "tests", "golden")

_G1 = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix(seed, n):
    """n 64-bit outputs of splitmix64 started at `seed` (counter form)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, n + 1, dtype=np.uint64) * _G1)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed, n):
    """doubles in [0, 1) with 53 random bits"""
    return (splitmix(seed, n) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def values(seed, n, kind, width=0):
    """kind: 'u' U[-1,1) | 'h' U[-0.5,0.5) | 'wide' U[-0.5,0.5) * 2^e, e uniform in [-width, width]
    | 'int' integers in [-1000, 1000] | 'maxmag' 1 - 2^-53 | 'sincos' exact-free smooth values"""
    if kind == "u":
        return 2.0 * uniform(seed, n) - 1.0
    if kind == "h":
        return uniform(seed, n) - 0.5
    if kind == "wide":
        e = (splitmix(seed ^ 0x5555, n) % np.uint64(2 * width + 1)).astype(np.int64) - width
        return np.ldexp(uniform(seed, n) - 0.5, e)
    if kind == "int":
        return (splitmix(seed, n) % np.uint64(2001)).astype(np.int64).astype(np.float64) - 1000.0
    if kind == "maxmag":
        return np.full(n, 1.0 - 2.0 ** -53)
    raise ValueError(kind)


def make_mat(seed, rows, cols, ld, kind, width=0, cplx=False, pad=1e300):
    """column-major (ld x cols) array; rows [rows, ld) hold `pad` so that stray reads show up
    (ref tests/test_ozaki2.cpp:49-50)"""
    dt = np.complex128 if cplx else np.float64
    X = np.full((ld, cols), pad, dtype=dt)
    if cplx:
        X[:rows] = (values(seed, rows * cols, kind, width) + 1j * values(seed + 7919, rows * cols, kind, width)
                    ).reshape(cols, rows).T
        X[rows:] = pad + 1j * pad
    else:
        X[:rows] = values(seed, rows * cols, kind, width).reshape(cols, rows).T
    return np.asfortranarray(X)


def op_shape(t, rows, cols):
    """(stored rows, stored cols) of X such that op(X) is rows x cols"""
    return (rows, cols) if t == "N" else (cols, rows)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def oracle():
    from pyoracle import Oracle
    o = Oracle()
    o.set_threads(os.cpu_count() or 1)
    return o


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def to_dev(a):
    """column-major numpy array -> CUDA tensor holding the same bytes (Fortran order kept)"""
    import torch
    flat = np.asfortranarray(a).ravel(order="F")
    if np.iscomplexobj(flat):
        flat = flat.view(np.float64)
    return torch.from_numpy(flat.copy()).cuda()


def from_dev(t, like):
    """CUDA tensor -> numpy array shaped like `like` (column-major)"""
    h = t.cpu().numpy()
    if np.iscomplexobj(like):
        h = h.view(np.complex128)
    return h.reshape(like.shape, order="F")
