"""The scale pass fused into the split against the separate passes and the oracle.

The fused kernel takes each plane row's maximum itself and writes it for the CRT, so every C must
be identical bit for bit with fusion on and off. Cases: both layouts (k contiguous up to k = 2048,
rows contiguous up to k = 1024), one side fused and the other not, the narrow and wide offsets,
non-finite and all-zero rows, a grouped call, and a tiled call (row panels of A split by separate
fused launches).
"""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def fusion():
    import oz2
    yield oz2
    oz2.set_scale_fusion(False)


def run(oz, ta, tb, m, n, k, s, A, B, C0, al=1.5, be=-0.5):
    import torch
    dC = to_dev(C0)
    oz.gemm(ta, tb, m, n, k, al, to_dev(A), A.shape[0], to_dev(B), B.shape[0], be, dC, C0.shape[0], s)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


CASES = [  # ta, tb, m, n, k, s
    ("T", "N", 300, 200, 2048, 16),  # both k contiguous, at the limit
    ("N", "T", 129, 257, 1024, 12),  # both rows contiguous, at the limit
    ("N", "N", 200, 150, 1500, 20),  # A rows contiguous beyond its limit (separate), B fused; wide offset
    ("T", "T", 77, 301, 40, 8),      # A fused (k contiguous), B rows contiguous fused
    ("N", "N", 1000, 30, 3000, 14),  # neither fused
]


@pytest.mark.parametrize("case", CASES)
def test_fused_scale_split_equals_separate_passes_and_the_oracle(oracle, oz, fusion, case):
    ta, tb, m, n, k, s = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(41 + s, Ar, Ac, Ar + 2, "wide", 25)
    B = make_mat(43 + s, Br, Bc, Br + 3, "wide", 25)
    C0 = make_mat(47 + s, m, n, m + 1, "u")
    fusion.set_scale_fusion(False)
    c_sep = run(oz, ta, tb, m, n, k, s, A, B, C0)
    fusion.set_scale_fusion(True)
    c_fused = run(oz, ta, tb, m, n, k, s, A, B, C0)
    assert np.array_equal(bits(c_fused), bits(c_sep)), f"{int((bits(c_fused) != bits(c_sep)).sum())} entries differ"
    want = C0.copy(order="F")
    assert oracle.dgemm(ta, tb, m, n, k, 1.5, A, Ar + 2, B, Br + 3, -0.5, want, m + 1, s) == 0
    assert np.array_equal(bits(c_fused), bits(want))


def test_non_finite_and_zero_rows(oracle, oz, fusion):
    m, n, k, s = 160, 150, 700, 15
    A = make_mat(1, k, m, k, "u")  # op(A) = A^T: k contiguous
    B = make_mat(2, k, n, k, "u")
    A[5, 9] = -np.inf
    A[:, 33] = 0.0
    B[100, 4] = np.nan
    B[:, 70] = 0.0
    C0 = make_mat(3, m, n, m, "u")
    out = {}
    for on in (False, True):
        fusion.set_scale_fusion(on)
        out[on] = run(oz, "T", "N", m, n, k, s, A, B, C0)
    assert np.array_equal(bits(out[True]), bits(out[False]))
    want = C0.copy(order="F")
    assert oracle.dgemm("T", "N", m, n, k, 1.5, A, k, B, k, -0.5, want, m, s) == 0
    assert np.array_equal(bits(out[True]), bits(want))
    assert np.isnan(out[True][9, :]).all() and np.isnan(out[True][:, 4]).all()


def test_grouped(oracle, oz, fusion):
    import torch
    specs = [("N", "N", 200, 130, 300, 16), ("T", "N", 64, 257, 2000, 16), ("N", "T", 129, 64, 900, 22),
             ("T", "T", 90, 100, 700, 9), ("N", "N", 300, 40, 5000, 12)]
    data = []
    for i, (ta, tb, m, n, k, s) in enumerate(specs):
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        data.append((make_mat(110 + i, Ar, Ac, Ar, "wide", 10), make_mat(120 + i, Br, Bc, Br, "wide", 10),
                     make_mat(130 + i, m, n, m, "u")))
    outs = {}
    for on in (False, True):
        fusion.set_scale_fusion(on)
        dev = [(to_dev(A), to_dev(B), to_dev(C0)) for A, B, C0 in data]
        probs = [(ta, tb, m, n, k, 1.0, dA, A.shape[0], dB, B.shape[0], 0.5, dC, m, s)
                 for (ta, tb, m, n, k, s), (A, B, _), (dA, dB, dC) in zip(specs, data, dev)]
        oz.gemm_grouped(probs)
        torch.cuda.synchronize()
        oz.check_device_error()
        outs[on] = [from_dev(dC, C0) for (_, _, dC), (_, _, C0) in zip(dev, data)]
    for i, ((ta, tb, m, n, k, s), (A, B, C0)) in enumerate(zip(specs, data)):
        assert np.array_equal(bits(outs[True][i]), bits(outs[False][i])), specs[i]
        want = C0.copy(order="F")
        assert oracle.dgemm(ta, tb, m, n, k, 1.0, A, A.shape[0], B, B.shape[0], 0.5, want, m, s) == 0
        assert np.array_equal(bits(outs[True][i]), bits(want)), specs[i]


def test_tiled_call(oracle, fusion):
    """a workspace limit that forces row and column panels: each panel's split is its own fused
    item, and the CRT of every tile reads maxima written by those launches"""
    import torch
    import oz2
    h = oz2.Ozaki2(torch.cuda.current_stream())
    try:
        m, n, k, s = 1200, 1100, 600, 14
        A = make_mat(7, k, m, k, "wide", 15)
        B = make_mat(8, k, n, k, "wide", 15)
        C0 = make_mat(9, m, n, m, "u")
        h.set_workspace_limit(24 << 20)
        out = {}
        for on in (False, True):
            fusion.set_scale_fusion(on)
            out[on] = run(h, "T", "N", m, n, k, s, A, B, C0)
        tiling = h.last_tiling()
        assert tiling.pm * tiling.pn > 1, tiling
        assert np.array_equal(bits(out[True]), bits(out[False]))
        want = C0.copy(order="F")
        assert oracle.dgemm("T", "N", m, n, k, 1.5, A, k, B, k, -0.5, want, m, s) == 0
        assert np.array_equal(bits(out[True]), bits(want))
    finally:
        h.close()
