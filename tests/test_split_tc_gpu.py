"""The tensor-core split against the integer-pipe (dp4a) split and the oracle.

Both kernels write the same residue planes, so every C they lead to must be identical bit for
bit; where the oracle finishes quickly the result is also checked against it. The cases cover the
three offset widths (two words: tk <= 62, three: tk <= 92, four: the extended sets), one and two
active TMEM lane quarters (s <= 16 and s > 16), both operand layouts (rows contiguous and k
contiguous), rows and k that are not multiples of the unit (16 x 32 or 4 x 128 elements), padded
leading dimensions, non-finite and all-zero rows, and a grouped call whose split launch holds
items with different s (the kernel rebuilds its weight tile between them).
"""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def split_kernels():
    import oz2
    yield oz2
    oz2.set_split_kernel(oz2.SPLIT_DEFAULT)


def run(oz, ta, tb, m, n, k, s, A, B, C0, al=1.5, be=-0.5):
    import torch
    dC = to_dev(C0)
    oz.gemm(ta, tb, m, n, k, al, to_dev(A), A.shape[0], to_dev(B), B.shape[0], be, dC, C0.shape[0], s)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


CASES = [  # ta, tb, m, n, k, s: tk from 8 (s = 3) to 88 (s = 24)
    ("N", "N", 300, 200, 777, 3),
    ("T", "N", 130, 257, 40, 8),
    ("N", "T", 129, 33, 1500, 12),
    ("T", "T", 200, 150, 300, 16),
    ("N", "N", 77, 301, 40, 17),   # tk 62: two words, two lane quarters
    ("N", "T", 260, 140, 777, 18),
    ("T", "N", 64, 90, 3000, 20),
    ("T", "T", 333, 129, 1000, 24),
]


@pytest.mark.parametrize("case", CASES)
def test_tensor_core_split_equals_the_dp4a_split_and_the_oracle(oracle, oz, split_kernels, case):
    ta, tb, m, n, k, s = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(11 + s, Ar, Ac, Ar + 3, "wide", 20)
    B = make_mat(23 + s, Br, Bc, Br + 1, "wide", 20)
    C0 = make_mat(37 + s, m, n, m + 2, "u")
    split_kernels.set_split_kernel(split_kernels.SPLIT_DP4A)
    c_int = run(oz, ta, tb, m, n, k, s, A, B, C0)
    split_kernels.set_split_kernel(split_kernels.SPLIT_TENSOR_CORE)
    c_tc = run(oz, ta, tb, m, n, k, s, A, B, C0)
    assert np.array_equal(bits(c_tc), bits(c_int)), f"{int((bits(c_tc) != bits(c_int)).sum())} entries differ"
    want = C0.copy(order="F")
    assert oracle.dgemm(ta, tb, m, n, k, 1.5, A, Ar + 3, B, Br + 1, -0.5, want, m + 2, s) == 0
    assert np.array_equal(bits(c_tc), bits(want))


def test_non_finite_and_zero_rows(oracle, oz, split_kernels):
    m, n, k, s = 150, 140, 500, 14
    A = make_mat(5, m, k, m, "u")
    B = make_mat(6, k, n, k, "u")
    A[3, 7] = np.inf
    A[40, :] = 0.0
    B[11, 9] = np.nan
    B[:, 100] = 0.0
    C0 = make_mat(7, m, n, m, "u")
    split_kernels.set_split_kernel(split_kernels.SPLIT_DP4A)
    c_int = run(oz, "N", "N", m, n, k, s, A, B, C0)
    split_kernels.set_split_kernel(split_kernels.SPLIT_TENSOR_CORE)
    c_tc = run(oz, "N", "N", m, n, k, s, A, B, C0)
    assert np.array_equal(bits(c_tc), bits(c_int))
    want = C0.copy(order="F")
    assert oracle.dgemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, want, m, s) == 0
    assert np.array_equal(bits(c_tc), bits(want))
    assert np.isnan(c_tc[3, :]).all() and np.isnan(c_tc[:, 9]).all()


def test_grouped_items_with_different_s(oracle, oz, split_kernels):
    """one split launch per layout and offset width holds items of several s: the weight tile
    and the lanes' moduli change between them"""
    import torch
    specs = [("N", "N", 200, 130, 300, 5), ("N", "N", 64, 257, 300, 16), ("N", "N", 129, 64, 300, 11),
             ("T", "T", 90, 100, 700, 17), ("T", "T", 300, 40, 700, 9)]
    data = []
    for i, (ta, tb, m, n, k, s) in enumerate(specs):
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        data.append((make_mat(50 + i, Ar, Ac, Ar, "wide", 10), make_mat(60 + i, Br, Bc, Br, "wide", 10),
                     make_mat(70 + i, m, n, m, "u")))
    outs = {}
    for kind in (split_kernels.SPLIT_DP4A, split_kernels.SPLIT_TENSOR_CORE):
        split_kernels.set_split_kernel(kind)
        dev = [(to_dev(A), to_dev(B), to_dev(C0)) for A, B, C0 in data]
        probs = [(ta, tb, m, n, k, 1.0, dA, A.shape[0], dB, B.shape[0], 0.5, dC, m, s)
                 for (ta, tb, m, n, k, s), (A, B, _), (dA, dB, dC) in zip(specs, data, dev)]
        oz.gemm_grouped(probs)
        torch.cuda.synchronize()
        oz.check_device_error()
        outs[kind] = [from_dev(dC, C0) for (_, _, dC), (_, _, C0) in zip(dev, data)]
    for i, ((ta, tb, m, n, k, s), (A, B, C0)) in enumerate(zip(specs, data)):
        got = outs[split_kernels.SPLIT_TENSOR_CORE][i]
        assert np.array_equal(bits(got), bits(outs[split_kernels.SPLIT_DP4A][i])), specs[i]
        want = C0.copy(order="F")
        assert oracle.dgemm(ta, tb, m, n, k, 1.0, A, A.shape[0], B, B.shape[0], 0.5, want, m, s) == 0
        assert np.array_equal(bits(got), bits(want)), specs[i]


@pytest.mark.parametrize("s", [26, 29, 32])
def test_extended_sets_four_word_offsets(oracle, split_kernels, s):
    """the adaptive path's extended moduli sets (tk up to 124: four-word offsets, moduli below
    128 from s = 29) through both split kernels"""
    import torch
    import oz2
    az = oz2.Ozaki2(torch.cuda.current_stream())
    try:
        ta, tb, m, n, k = ("T", "N", 130, 257, 1500) if s != 29 else ("N", "T", 300, 200, 777)
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        A = make_mat(100 + s, Ar, Ac, Ar + 2, "wide", 30)
        B = make_mat(200 + s, Br, Bc, Br + 1, "wide", 30)
        C0 = make_mat(300 + s, m, n, m + 3, "u")
        got = {}
        for kind in (split_kernels.SPLIT_DP4A, split_kernels.SPLIT_TENSOR_CORE):
            split_kernels.set_split_kernel(kind)
            dC = to_dev(C0)
            az.gemm_adaptive([(ta, tb, m, n, k, 1.5, to_dev(A), Ar + 2, to_dev(B), Br + 1, -0.5, dC, m + 3, s)], 53,
                             az.ADAPTIVE_FIXED)
            torch.cuda.synchronize()
            az.check_device_error()
            got[kind] = from_dev(dC, C0)
        assert np.array_equal(bits(got[1]), bits(got[0]))
        want = C0.copy(order="F")
        assert oracle.dgemm_ext(ta, tb, m, n, k, 1.5, A, Ar + 2, B, Br + 1, -0.5, want, m + 3, s) == 0
        assert np.array_equal(bits(got[1]), bits(want))
    finally:
        az.close()


def test_split_kernel_selector_is_checked(split_kernels):
    with pytest.raises(ValueError):
        split_kernels.set_split_kernel(2)
