"""The tensor-core CRT against the dp2a CRT and the oracle.

Both kernels reconstruct from the same residues with the same carry chain and rounding, so every
C must be identical bit for bit. The cases cover every limb count (2 to 8 limbs: s = 2 .. 32, the
extended sets through the adaptive path's fixed-s mode), beta zero and non-zero, m not a multiple
of the 32-row super-tile, n not a multiple of its 16 columns, padded leading dimensions,
non-finite rows and columns, and a grouped call with several s.
"""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def crt_kernels():
    import oz2
    yield oz2
    oz2.set_crt_kernel(oz2.CRT_DEFAULT)


def run(oz, ta, tb, m, n, k, s, A, B, C0, al, be):
    import torch
    dC = to_dev(C0)
    oz.gemm(ta, tb, m, n, k, al, to_dev(A), A.shape[0], to_dev(B), B.shape[0], be, dC, C0.shape[0], s)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


CASES = [  # ta, tb, m, n, k, s, beta: limbs 2, 2, 3, 4, 4, 5, 6, 6
    ("N", "N", 100, 70, 300, 2, 0.0),
    ("T", "N", 33, 17, 1000, 8, -0.5),
    ("N", "T", 257, 129, 500, 11, 0.0),
    ("T", "T", 64, 48, 64, 13, 2.0),
    ("N", "N", 300, 200, 777, 16, -0.5),
    ("N", "T", 31, 300, 1500, 19, 0.0),
    ("T", "N", 129, 65, 3000, 22, -1.0),
    ("T", "T", 200, 15, 2000, 24, 0.5),
]


@pytest.mark.parametrize("case", CASES)
def test_tensor_core_crt_equals_the_dp2a_crt_and_the_oracle(oracle, oz, crt_kernels, case):
    ta, tb, m, n, k, s, be = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(3 + s, Ar, Ac, Ar + 1, "wide", 25)
    B = make_mat(9 + s, Br, Bc, Br + 2, "wide", 25)
    C0 = make_mat(17 + s, m, n, m + 5, "u")
    crt_kernels.set_crt_kernel(crt_kernels.CRT_DP2A)
    c_dp = run(oz, ta, tb, m, n, k, s, A, B, C0, 1.25, be)
    crt_kernels.set_crt_kernel(crt_kernels.CRT_TENSOR_CORE)
    c_tc = run(oz, ta, tb, m, n, k, s, A, B, C0, 1.25, be)
    assert np.array_equal(bits(c_tc), bits(c_dp)), f"{int((bits(c_tc) != bits(c_dp)).sum())} entries differ"
    want = C0.copy(order="F")
    assert oracle.dgemm(ta, tb, m, n, k, 1.25, A, Ar + 1, B, Br + 2, be, want, m + 5, s) == 0
    assert np.array_equal(bits(c_tc), bits(want))


def test_non_finite_rows_and_columns(oracle, oz, crt_kernels):
    m, n, k, s = 150, 140, 500, 18
    A = make_mat(5, m, k, m, "u")
    B = make_mat(6, k, n, k, "u")
    A[3, 7] = np.inf
    A[40, :] = 0.0
    B[11, 9] = np.nan
    C0 = make_mat(7, m, n, m, "u")
    out = {}
    for kind in (crt_kernels.CRT_DP2A, crt_kernels.CRT_TENSOR_CORE):
        crt_kernels.set_crt_kernel(kind)
        out[kind] = run(oz, "N", "N", m, n, k, s, A, B, C0, 1.5, -0.5)
    assert np.array_equal(bits(out[1]), bits(out[0]))
    want = C0.copy(order="F")
    assert oracle.dgemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, want, m, s) == 0
    assert np.array_equal(bits(out[1]), bits(want))
    assert np.isnan(out[1][3, :]).all() and np.isnan(out[1][:, 9]).all()


def test_grouped_problems(oracle, oz, crt_kernels):
    import torch
    specs = [("N", "N", 200, 130, 300, 14), ("N", "T", 64, 257, 300, 14), ("T", "N", 129, 64, 300, 20),
             ("T", "T", 90, 100, 700, 20), ("N", "N", 300, 40, 700, 9)]
    data = []
    for i, (ta, tb, m, n, k, s) in enumerate(specs):
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        data.append((make_mat(80 + i, Ar, Ac, Ar, "wide", 10), make_mat(90 + i, Br, Bc, Br, "wide", 10),
                     make_mat(99 + i, m, n, m, "u")))
    outs = {}
    for kind in (crt_kernels.CRT_DP2A, crt_kernels.CRT_TENSOR_CORE):
        crt_kernels.set_crt_kernel(kind)
        dev = [(to_dev(A), to_dev(B), to_dev(C0)) for A, B, C0 in data]
        probs = [(ta, tb, m, n, k, 1.0, dA, A.shape[0], dB, B.shape[0], 0.5, dC, m, s)
                 for (ta, tb, m, n, k, s), (A, B, _), (dA, dB, dC) in zip(specs, data, dev)]
        oz.gemm_grouped(probs)
        torch.cuda.synchronize()
        oz.check_device_error()
        outs[kind] = [from_dev(dC, C0) for (_, _, dC), (_, _, C0) in zip(dev, data)]
    for i, ((ta, tb, m, n, k, s), (A, B, C0)) in enumerate(zip(specs, data)):
        got = outs[crt_kernels.CRT_TENSOR_CORE][i]
        assert np.array_equal(bits(got), bits(outs[crt_kernels.CRT_DP2A][i])), specs[i]
        want = C0.copy(order="F")
        assert oracle.dgemm(ta, tb, m, n, k, 1.0, A, A.shape[0], B, B.shape[0], 0.5, want, m, s) == 0
        assert np.array_equal(bits(got), bits(want)), specs[i]


@pytest.mark.parametrize("s", [26, 30])
def test_extended_sets(oracle, crt_kernels, s):
    """7 and 8 limbs (the adaptive path's extended moduli sets)"""
    import torch
    import oz2
    az = oz2.Ozaki2(torch.cuda.current_stream())
    try:
        ta, tb, m, n, k = "N", "T", 300, 200, 777
        A = make_mat(100 + s, m, k, m + 2, "wide", 30)
        B = make_mat(200 + s, n, k, n + 1, "wide", 30)
        C0 = make_mat(300 + s, m, n, m + 3, "u")
        got = {}
        for kind in (crt_kernels.CRT_DP2A, crt_kernels.CRT_TENSOR_CORE):
            crt_kernels.set_crt_kernel(kind)
            dC = to_dev(C0)
            az.gemm_adaptive([(ta, tb, m, n, k, 1.5, to_dev(A), m + 2, to_dev(B), n + 1, -0.5, dC, m + 3, s)], 53,
                             az.ADAPTIVE_FIXED)
            torch.cuda.synchronize()
            az.check_device_error()
            got[kind] = from_dev(dC, C0)
        assert np.array_equal(bits(got[1]), bits(got[0]))
        want = C0.copy(order="F")
        assert oracle.dgemm_ext(ta, tb, m, n, k, 1.5, A, m + 2, B, n + 1, -0.5, want, m + 3, s) == 0
        assert np.array_equal(bits(got[1]), bits(want))
    finally:
        az.close()
