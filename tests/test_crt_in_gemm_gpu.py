"""The CRT in the GEMM's epilogue (s <= 8) against the separate CRT launch and the oracle.

With the fusion on, a real problem of s <= 8 and k <= 65408 keeps each tile's residues in tensor
memory and its GEMM writes C; every C must equal, bit for bit, the one from residue planes and a
separate CRT launch, and the oracle's. Cases: every s from 2 to 8, m and n not multiples of the
128 x 128 tile, alpha / beta, padded ldc, non-finite rows and columns, the largest fused k and the
first k beyond it, a tiled call, and a grouped call mixing fused and unfused problems.
"""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def crt_fusion():
    import oz2
    yield oz2
    oz2.set_crt_fusion(False)


def run(oz, ta, tb, m, n, k, s, A, B, C0, al, be):
    import torch
    dC = to_dev(C0)
    oz.gemm(ta, tb, m, n, k, al, to_dev(A), A.shape[0], to_dev(B), B.shape[0], be, dC, C0.shape[0], s)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


def both(oz, crt_fusion, *args):
    out = {}
    for on in (False, True):
        crt_fusion.set_crt_fusion(on)
        out[on] = run(oz, *args)
    return out


CASES = [  # ta, tb, m, n, k, s, alpha, beta
    ("N", "N", 300, 200, 777, 2, 1.0, 0.0),
    ("T", "N", 129, 257, 1500, 3, 1.5, -0.5),
    ("N", "T", 128, 128, 64, 4, -2.0, 1.0),
    ("T", "T", 77, 301, 3000, 5, 0.75, 0.0),
    ("N", "N", 513, 130, 200, 6, 1.0, 0.25),
    ("T", "N", 256, 129, 40, 7, 3.0, -1.0),
    ("N", "T", 600, 500, 400, 8, 1.5, -0.5),
]


@pytest.mark.parametrize("case", CASES)
def test_crt_in_gemm_equals_the_crt_launch_and_the_oracle(oracle, oz, crt_fusion, case):
    ta, tb, m, n, k, s, al, be = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(61 + s, Ar, Ac, Ar + 1, "wide", 6)
    B = make_mat(67 + s, Br, Bc, Br + 2, "wide", 6)
    C0 = make_mat(71 + s, m, n, m + 3, "u")
    out = both(oz, crt_fusion, ta, tb, m, n, k, s, A, B, C0, al, be)
    assert np.array_equal(bits(out[True]), bits(out[False])), f"{int((bits(out[True]) != bits(out[False])).sum())} differ"
    want = C0.copy(order="F")
    assert oracle.dgemm(ta, tb, m, n, k, al, A, Ar + 1, B, Br + 2, be, want, m + 3, s) == 0
    assert np.array_equal(bits(out[True]), bits(want))


def test_non_finite_rows_and_columns(oracle, oz, crt_fusion):
    m, n, k, s = 200, 190, 300, 8
    A = make_mat(1, m, k, m, "u")
    B = make_mat(2, k, n, k, "u")
    A[17, 5] = np.nan
    A[60, :] = 0.0
    B[9, 150] = -np.inf
    C0 = make_mat(3, m, n, m, "u")
    out = both(oz, crt_fusion, "N", "N", m, n, k, s, A, B, C0, 1.5, -0.5)
    assert np.array_equal(bits(out[True]), bits(out[False]))
    want = C0.copy(order="F")
    assert oracle.dgemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, want, m, s) == 0
    assert np.array_equal(bits(out[True]), bits(want))
    assert np.isnan(out[True][17, :]).all() and np.isnan(out[True][:, 150]).all()


@pytest.mark.parametrize("k", [65408, 65409])
def test_the_k_limit(oracle, oz, crt_fusion, k):
    """65408 = 511 k blocks (the exact quotient's limit) is fused, 65409 runs the CRT launch"""
    m, n, s = 70, 40, 8
    A = make_mat(4, m, k, m, "h")
    B = make_mat(5, k, n, k, "h")
    C0 = make_mat(6, m, n, m, "u")
    out = both(oz, crt_fusion, "N", "N", m, n, k, s, A, B, C0, 1.0, 0.5)
    assert np.array_equal(bits(out[True]), bits(out[False]))
    want = C0.copy(order="F")
    assert oracle.dgemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.5, want, m, s) == 0
    assert np.array_equal(bits(out[True]), bits(want))


def test_tiled_call(oracle, crt_fusion):
    import torch
    import oz2
    h = oz2.Ozaki2(torch.cuda.current_stream())
    try:
        m, n, k, s = 1500, 1300, 700, 6
        A = make_mat(7, k, m, k, "wide", 10)
        B = make_mat(8, k, n, k, "wide", 10)
        C0 = make_mat(9, m, n, m + 7, "u")
        h.set_workspace_limit(24 << 20)
        out = both(h, crt_fusion, "T", "N", m, n, k, s, A, B, C0, 1.5, -0.5)
        tiling = h.last_tiling()
        assert tiling.pm * tiling.pn > 1, tiling
        assert np.array_equal(bits(out[True]), bits(out[False]))
        want = C0.copy(order="F")
        assert oracle.dgemm("T", "N", m, n, k, 1.5, A, k, B, k, -0.5, want, m + 7, s) == 0
        assert np.array_equal(bits(out[True]), bits(want))
    finally:
        h.close()


def test_grouped_mixed(oracle, oz, crt_fusion):
    """fused problems (s <= 8, one launch per s) beside unfused ones (s > 8, the CRT launches)"""
    import torch
    specs = [("N", "N", 200, 130, 300, 8), ("T", "N", 64, 257, 2000, 16), ("N", "T", 129, 64, 900, 4),
             ("T", "T", 90, 100, 700, 8), ("N", "N", 300, 40, 500, 12), ("N", "N", 33, 33, 33, 2)]
    data = []
    for i, (ta, tb, m, n, k, s) in enumerate(specs):
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        data.append((make_mat(140 + i, Ar, Ac, Ar, "wide", 8), make_mat(150 + i, Br, Bc, Br, "wide", 8),
                     make_mat(160 + i, m, n, m, "u")))
    outs = {}
    for on in (False, True):
        crt_fusion.set_crt_fusion(on)
        dev = [(to_dev(A), to_dev(B), to_dev(C0)) for A, B, C0 in data]
        probs = [(ta, tb, m, n, k, 1.25, dA, A.shape[0], dB, B.shape[0], -0.75, dC, m, s)
                 for (ta, tb, m, n, k, s), (A, B, _), (dA, dB, dC) in zip(specs, data, dev)]
        oz.gemm_grouped(probs)
        torch.cuda.synchronize()
        oz.check_device_error()
        outs[on] = [from_dev(dC, C0) for (_, _, dC), (_, _, C0) in zip(dev, data)]
    for i, ((ta, tb, m, n, k, s), (A, B, C0)) in enumerate(zip(specs, data)):
        assert np.array_equal(bits(outs[True][i]), bits(outs[False][i])), specs[i]
        want = C0.copy(order="F")
        assert oracle.dgemm(ta, tb, m, n, k, 1.25, A, A.shape[0], B, B.shape[0], -0.75, want, m, s) == 0
        assert np.array_equal(bits(outs[True][i]), bits(want)), specs[i]
