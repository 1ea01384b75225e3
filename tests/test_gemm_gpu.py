"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Bit-exact: every case compares the GPU result with the reference's own output (golden
fixtures) or with the oracle, which is pinned to the reference. The reference's rigorous
element-wise bound against a double-double product (tests/test_ozaki2.cpp:155-178) is checked
as well, and rows m..ldc of C must stay untouched.
"""
import os

import numpy as np
import pytest

from common import GOLDEN, bits, from_dev, make_mat, op_shape, to_dev
from make_golden import DGEMM_CASES, ZGEMM_CASES, dgemm_inputs, zgemm_inputs

pytestmark = pytest.mark.gpu


def run_dgemm(oz, ta, tb, m, n, k, al, A, B, be, C0, s):
    import torch
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    oz.gemm(ta, tb, m, n, k, al, dA, A.shape[0], dB, B.shape[0], be, dC, C0.shape[0], s)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


def run_zgemm(oz, ta, tb, m, n, k, al, A, B, be, C0, s):
    import torch
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    oz.zgemm(ta, tb, m, n, k, al, dA, A.shape[0], dB, B.shape[0], be, dC, C0.shape[0], s)
    torch.cuda.synchronize()
    oz.check_device_error()
    return from_dev(dC, C0)


def check_against_oracle(oracle, oz, ta, tb, m, n, k, s, al, be, A, B, C0, bound=True):
    C = run_dgemm(oz, ta, tb, m, n, k, al, A, B, be, C0, s)
    Co = C0.copy(order="F")
    assert oracle.dgemm(ta, tb, m, n, k, al, A, A.shape[0], B, B.shape[0], be, Co, C0.shape[0], s) == 0
    nd = int((bits(C) != bits(Co)).sum())
    assert nd == 0, f"{nd} entries differ from the oracle"
    if bound:
        hi, lo = oracle.dd_gemm(ta, tb, m, n, k, A, A.shape[0], B, B.shape[0])
        r = oracle.bound_ratio(ta, tb, m, n, k, s, A, A.shape[0], B, B.shape[0], al, be, C0, C, C0.shape[0], hi, lo)
        assert r <= 1.0, r
    return C


@pytest.mark.parametrize("ci", range(len(DGEMM_CASES)))
def test_dgemm_golden(oz, ci):
    g = np.load(os.path.join(GOLDEN, "dgemm_cases.npz"))
    case = DGEMM_CASES[ci]
    ta, tb, m, n, k, s, al, be = case[:8]
    A, B, C0 = dgemm_inputs(case)
    C = run_dgemm(oz, ta, tb, m, n, k, al, A, B, be, C0, s)
    assert np.array_equal(bits(C), bits(g[f"C{ci}"])), case


@pytest.mark.parametrize("ci", range(len(ZGEMM_CASES)))
def test_zgemm_golden(oz, ci):
    g = np.load(os.path.join(GOLDEN, "zgemm_cases.npz"))
    case = ZGEMM_CASES[ci]
    ta, tb, m, n, k, s, al, be = case[:8]
    A, B, C0 = zgemm_inputs(case)
    C = run_zgemm(oz, ta, tb, m, n, k, al, A, B, be, C0, s)
    assert np.array_equal(bits(C), bits(g[f"C{ci}"])), case


@pytest.mark.parametrize("s", range(2, 25))
def test_accuracy_vs_s(oracle, oz, s):
    """ref tests/test_ozaki2.cpp:448-452: 256 x 256 x 1024 for every s (s too small -> error)"""
    m = n = 256
    k = 1024
    A = make_mat(500 + s, m, k, m, "wide", 3)
    B = make_mat(600 + s, k, n, k, "wide", 3)
    C0 = make_mat(700, m, n, m, "u")
    try:
        oracle.plan(s, k)
    except ValueError:
        with pytest.raises(ValueError):
            run_dgemm(oz, "N", "N", m, n, k, 1.0, A, B, 0.0, C0, s)
        return
    check_against_oracle(oracle, oz, "N", "N", m, n, k, s, 1.0, 0.0, A, B, C0)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", [(1, 1, 1), (37, 53, 129), (130, 7, 1), (257, 129, 130), (300, 520, 700)])
def test_shapes_and_ops(oracle, oz, ta, tb, shape):
    m, n, k = shape
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(800 + m, Ar, Ac, Ar + 3, "wide", 5)
    B = make_mat(900 + n, Br, Bc, Br + 1, "wide", 5)
    C0 = make_mat(1000, m, n, m + 5, "u")
    check_against_oracle(oracle, oz, ta, tb, m, n, k, 14, -1.5, 0.25, A, B, C0)


def test_wide_path_and_exact_integers(oracle, oz):
    for s, kind, width in [(20, "wide", 30), (24, "wide", 40), (12, "int", 0)]:
        A = make_mat(1100 + s, 96, 640, 96, kind, width)
        B = make_mat(1200 + s, 640, 72, 640, kind, width)
        C0 = np.zeros((96, 72), order="F")
        C = check_against_oracle(oracle, oz, "N", "N", 96, 72, 640, s, 1.0, 0.0, A, B, C0)
        if kind == "int":
            assert np.array_equal(C, A @ B)  # exact products of integers are exact


@pytest.mark.parametrize("s", [3, 4, 8, 12, 16, 20, 24])
def test_max_magnitude(oracle, oz, s):
    """|C'| ~ M/4 (ref tests/test_ozaki2.cpp:470-471)"""
    A = make_mat(1, 64, 4096, 64, "maxmag")
    B = make_mat(2, 4096, 64, 4096, "maxmag")
    check_against_oracle(oracle, oz, "N", "N", 64, 64, 4096, s, 1.0, 0.0, A, B, np.zeros((64, 64), order="F"))


def test_tiling_bit_identical(oracle, oz):
    """ref tests/test_ozaki2.cpp:473-486: an 8 MiB workspace limit forces C tiles; the result
    must equal the one-tile result bit for bit"""
    m, n, k = 1000, 900, 512
    A = make_mat(31, m, k, m, "wide", 4)
    B = make_mat(32, n, k, n, "wide", 4)
    C0 = np.zeros((m, n), order="F")
    C1 = run_dgemm(oz, "N", "T", m, n, k, 1.0, A, B, 0.0, C0, 10)
    t1 = oz.last_tiling()
    oz.set_workspace_limit(8 << 20)
    try:
        C2 = run_dgemm(oz, "N", "T", m, n, k, 1.0, A, B, 0.0, C0, 10)
        t2 = oz.last_tiling()
    finally:
        oz.set_workspace_limit(0)
    assert t1.pm * t1.pn == 1 and t2.pm * t2.pn > 1
    assert t2.workspace_bytes <= 8 << 20
    assert np.array_equal(bits(C1), bits(C2))
    Co = C0.copy(order="F")
    oracle.dgemm("N", "T", m, n, k, 1.0, A, m, B, n, 0.0, Co, m, 10)
    assert np.array_equal(bits(C1), bits(Co))


@pytest.mark.parametrize("ta,m,n,k", [("N", 16, 24, 300000), ("T", 8, 8, 140000)])
def test_k_chunks(oracle, oz, ta, m, n, k):
    """k beyond the exact int32 range of one product (ref tests/test_ozaki2.cpp:488-489)"""
    Ar, Ac = op_shape(ta, m, k)
    A = make_mat(41, Ar, Ac, Ar, "wide", 2)
    B = make_mat(42, k, n, k, "wide", 2)
    C = check_against_oracle(oracle, oz, ta, "N", m, n, k, 18, 1.0, 0.0, A, B, np.zeros((m, n), order="F"))
    assert oz.last_tiling().k_chunks >= 2


def test_nonfinite_propagation(oz):
    m, n, k = 32, 32, 64
    A = np.full((m, k), 0.5, order="F")
    B = np.full((k, n), 0.25, order="F")
    A[3, 10] = np.inf
    B[5, 7] = np.nan
    C = run_dgemm(oz, "N", "N", m, n, k, 1.0, A, B, 0.0, np.zeros((m, n), order="F"), 8)
    nan = np.isnan(C)
    assert nan[3].all() and nan[:, 7].all() and nan.sum() == m + n - 1
    assert (C[~nan] == 0.5 * 0.25 * k).all()


def test_subnormal_results(oracle, oz):
    """results that land in the subnormal range go through the same final ldexp rounding"""
    A = make_mat(51, 64, 128, 64, "h") * 2.0 ** -520
    B = make_mat(52, 128, 64, 128, "h") * 2.0 ** -530
    check_against_oracle(oracle, oz, "N", "N", 64, 64, 128, 16, 1.0, 0.0, np.asfortranarray(A),
                         np.asfortranarray(B), np.zeros((64, 64), order="F"), bound=False)


def test_errors_and_early_returns(oz):
    import torch
    d = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="negative dimension"):
        oz.gemm("N", "N", -1, 4, 4, 1.0, d, 4, d, 4, 0.0, d, 4, 8)
    with pytest.raises(ValueError, match="leading dimension"):
        oz.gemm("N", "N", 4, 4, 4, 1.0, d, 3, d, 4, 0.0, d, 4, 8)
    with pytest.raises(ValueError, match="num_moduli"):
        oz.gemm("N", "N", 4, 4, 4, 1.0, d, 4, d, 4, 0.0, d, 4, 25)
    with pytest.raises(ValueError, match="too small"):
        oz.gemm("N", "N", 4, 4, 10 ** 6, 1.0, d, 4, d, 10 ** 6, 0.0, d, 4, 2)
    oz.gemm("N", "N", 0, 4, 4, 1.0, d, 4, d, 4, 0.0, d, 4, 99)  # m == 0: no check of s
    c = torch.arange(16, dtype=torch.float64, device="cuda")
    oz.gemm("N", "N", 4, 4, 0, 1.0, d, 4, d, 4, 0.5, c, 4, 8)  # k == 0: C = beta C
    torch.cuda.synchronize()
    assert torch.equal(c.cpu(), torch.arange(16, dtype=torch.float64) * 0.5)
    oz.gemm("N", "N", 4, 4, 4, 0.0, d, 4, d, 4, 0.0, c, 4, 8)  # alpha == 0, beta == 0: zeros
    torch.cuda.synchronize()
    assert not c.any()


def test_stage_times_and_tiling(oz):
    import torch
    m = n = k = 512
    A = to_dev(make_mat(61, m, k, m, "h"))
    B = to_dev(make_mat(62, k, n, k, "h"))
    C = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    oz.set_profiling(True)
    try:
        oz.gemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, 16)
        st = oz.stage_times()
    finally:
        oz.set_profiling(False)
    assert st.scale_ms > 0 and st.split_ms > 0 and st.gemm_ms > 0 and st.crt_ms > 0
    t = oz.last_tiling()
    assert (t.mb, t.nb, t.pm, t.pn, t.k_chunks) == (512, 512, 1, 1, 1) and t.workspace_bytes > 0
