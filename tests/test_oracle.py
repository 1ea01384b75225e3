"""The C oracle against the golden vectors of the reference and against restated known-answer
tests of the reference's own suite (tests/test_ozaki2.cpp). CPU only."""
import json
import os
import subprocess

import numpy as np
import pytest

from common import GOLDEN, ROOT, bits, make_mat, op_shape
from make_golden import DGEMM_CASES, SPLIT_CASES, ZGEMM_CASES, dgemm_inputs, zgemm_inputs


def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


def test_plans_match_reference(oracle):
    data = json.load(open(os.path.join(GOLDEN, "plans.json")))
    for e in data["plans"]:
        if e.get("invalid"):
            with pytest.raises(ValueError):
                oracle.plan(e["s"], e["k"])
            continue
        p = oracle.plan(e["s"], e["k"])
        assert (p.tk, p.nl, p.log2M) == (e["tk"], e["nl"], e["log2M"]), e
        assert p.Mint == int(e["M"], 16)
        for t in range(e["s"]):
            assert (p.m[t], p.y[t], p.Wint(t)) == (e["m"][t], e["y"][t], int(e["W"][t], 16))
    for key, s in data["moduli_for_bits"].items():
        k, b = map(int, key.split(":"))
        assert oracle.moduli_for_bits(k, b) == s, key


@pytest.mark.parametrize("s,tk", SPLIT_CASES)
def test_split_matches_reference(oracle, s, tk):
    g = _golden(f"split_s{s}_tk{tk}.npz")
    P = oracle.split(g["X"], g["ex"], False, oracle.plan(s, 16))
    assert np.array_equal(P, g["P"])


@pytest.mark.parametrize("s,tk", SPLIT_CASES)
def test_split_known_answer(oracle, s, tk):
    """independent exact scaling and symmetric residue in Python integers, as the reference's
    unit_split does with __int128 (tests/test_ozaki2.cpp:195-254)"""
    g = _golden(f"split_s{s}_tk{tk}.npz")
    X, ex = g["X"], g["ex"]
    p = oracle.plan(s, 16)
    P = oracle.split(X, ex, False, p)
    bad = 0
    for c in range(X.shape[1]):
        for r in range(X.shape[0]):
            v = float(X[r, c])
            if v == 0.0:
                x = 0
            else:
                fr, qe = np.frexp(abs(v))
                mant = int(np.ldexp(fr, 53))
                sh = int(qe) - 53 + int(ex[c])
                if sh >= 0:
                    x = mant << sh
                elif sh < -60:
                    x = 0
                else:
                    q, rem, half = mant >> -sh, mant & ((1 << -sh) - 1), 1 << (-sh - 1)
                    x = q + (1 if rem > half or (rem == half and q & 1) else 0)
                if v < 0:
                    x = -x
            for t in range(s):
                m = p.m[t]
                h = (m - 1) // 2
                rr = (x + h) % m - h
                bad += np.int8(np.uint8(rr & 0xFF)) != P[t, c, r]
    assert bad == 0


def test_crt_matches_reference(oracle):
    g = _golden("crt_cases.npz")
    for s in range(2, 25):
        p = oracle.plan(s, 16)
        Ct, D, out = g[f"Ct{s}"], g[f"D{s}"], g[f"out{s}"]
        got = np.array([oracle.crt(p, Ct[:, i].astype(np.int64), int(D[i]) + 3) for i in range(Ct.shape[1])])
        assert np.array_equal(bits(got), bits(out)), s


def _big_to_double_rne(x, scale):
    """restates tests/test_ozaki2.cpp:256-270"""
    neg = x < 0
    x = abs(x)
    if x == 0:
        return 0.0
    top = x.bit_length() - 1
    if top >= 53:
        rb = top - 53
        m53 = x >> (rb + 1)
        rnd = (x >> rb) & 1
        sticky = x & ((1 << rb) - 1)
        if rnd and (sticky or (m53 & 1)):
            m53 += 1
        v = float(np.ldexp(float(m53), top - 52 + scale))
    else:
        v = float(np.ldexp(float(x), scale))
    return -v if neg else v


def test_crt_known_answer(oracle):
    rng = np.random.default_rng(5)
    for s in (2, 7, 13, 16, 20, 24):
        p = oracle.plan(s, 16)
        Mq = p.Mint // 4
        for i in range(300):
            x = min(int.from_bytes(rng.bytes(32), "little") % (Mq + 1), Mq) if i else Mq
            if rng.integers(0, 2):
                x = -x
            shift = int(rng.integers(-20, 21))
            r = [x % p.m[t] + int(rng.integers(-1000, 1000)) * p.m[t] for t in range(s)]
            got = oracle.crt(p, np.array(r, np.int64), shift)
            assert got == _big_to_double_rne(x, -shift) or (got == 0 and x == 0), (s, x)


def test_dgemm_matches_reference(oracle):
    g = _golden("dgemm_cases.npz")
    for ci, case in enumerate(DGEMM_CASES):
        ta, tb, m, n, k, s, al, be = case[:8]
        A, B, C0 = dgemm_inputs(case)
        C = C0.copy(order="F")
        assert oracle.dgemm(ta, tb, m, n, k, al, A, A.shape[0], B, B.shape[0], be, C, C.shape[0], s) == 0
        assert np.array_equal(bits(C), bits(g[f"C{ci}"])), case
        hi, lo = oracle.dd_gemm(ta, tb, m, n, k, A, A.shape[0], B, B.shape[0])
        assert oracle.bound_ratio(ta, tb, m, n, k, s, A, A.shape[0], B, B.shape[0], al, be, C0, C, C.shape[0], hi,
                                  lo) <= 1.0, case
        assert np.array_equal(bits(C[m:]), bits(C0[m:]))  # rows m..ldc untouched


def test_zgemm_matches_reference(oracle):
    g = _golden("zgemm_cases.npz")
    for ci, case in enumerate(ZGEMM_CASES):
        ta, tb, m, n, k, s, al, be = case[:8]
        A, B, C0 = zgemm_inputs(case)
        C = C0.copy(order="F")
        assert oracle.zgemm(ta, tb, m, n, k, al, A, A.shape[0], B, B.shape[0], be, C, C.shape[0], s) == 0
        assert np.array_equal(bits(C), bits(g[f"C{ci}"])), case
        hi, lo = oracle.dd_zgemm(ta, tb, m, n, k, A, A.shape[0], B, B.shape[0])
        assert oracle.zbound_ratio(ta, tb, m, n, k, s, A, A.shape[0], B, B.shape[0], al, be, C0, C, C.shape[0], hi,
                                   lo) <= 1.0, case


def test_nonfinite_propagation(oracle):
    """ref tests/test_ozaki2.cpp:522-543: Inf in A(3,10), NaN in B(5,7) -> NaN exactly on row 3
    and column 7, 0.5 * 0.25 * k elsewhere"""
    m, n, k = 32, 32, 64
    A = np.full((m, k), 0.5, order="F")
    B = np.full((k, n), 0.25, order="F")
    A[3, 10] = np.inf
    B[5, 7] = np.nan
    C = np.zeros((m, n), order="F")
    assert oracle.dgemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, 8) == 0
    nan = np.isnan(C)
    assert nan[3].all() and nan[:, 7].all() and nan.sum() == m + n - 1
    assert (C[~nan] == 0.5 * 0.25 * k).all()


def test_invalid_arguments(oracle):
    A = np.zeros((4, 4), order="F")
    assert oracle.dgemm("N", "N", -1, 4, 4, 1.0, A, 4, A, 4, 0.0, A, 4, 8) == 1
    assert oracle.dgemm("N", "N", 4, 4, 4, 1.0, A, 3, A, 4, 0.0, A, 4, 8) == 1
    assert oracle.dgemm("N", "N", 4, 4, 4, 1.0, A, 4, A, 4, 0.0, A, 4, 25) == 1
    assert oracle.dgemm("N", "N", 4, 4, 4, 1.0, A, 4, A, 4, 0.0, A, 4, 1) == 1
    # m == 0 returns before the number of moduli is checked (ref src/ozaki2_gpu.hpp:750)
    assert oracle.dgemm("N", "N", 0, 4, 4, 1.0, A, 4, A, 4, 0.0, A, 4, 99) == 0


def test_oracle_against_reference_build(oracle, ref):
    """random shapes through both CPU paths (the reference built here and the oracle)"""
    rng = np.random.default_rng(99)
    for trial in range(6):
        ta, tb = rng.choice(list("NT")), rng.choice(list("NT"))
        m, n, k = (int(x) for x in rng.integers(1, 90, 3))
        s = int(rng.integers(6, 25))
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        A = make_mat(100 + trial, Ar, Ac, Ar + 2, "wide", 8)
        B = make_mat(200 + trial, Br, Bc, Br + 1, "wide", 8)
        C1 = make_mat(300 + trial, m, n, m + 3, "u")
        C2 = C1.copy(order="F")
        st_o = oracle.dgemm(ta, tb, m, n, k, 0.75, A, Ar + 2, B, Br + 1, -2.0, C1, m + 3, s)
        st_r, _ = ref.dgemm(ta, tb, m, n, k, 0.75, A, Ar + 2, B, Br + 1, -2.0, C2, m + 3, s)
        assert st_o == st_r
        assert np.array_equal(bits(C1), bits(C2)), (ta, tb, m, n, k, s)


def test_zgemm_oracle_against_reference_build(oracle, ref):
    """random complex products through both CPU paths: every op pair, s across the narrow and wide
    paths (the plan of 2k), alpha and beta complex"""
    rng = np.random.default_rng(123)
    for trial in range(8):
        ta, tb = rng.choice(list("NTC")), rng.choice(list("NTC"))
        m, n, k = (int(x) for x in rng.integers(1, 60, 3))
        s = int(rng.integers(6, 25))
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        A = make_mat(400 + trial, Ar, Ac, Ar + 1, "wide", 10, cplx=True)
        B = make_mat(500 + trial, Br, Bc, Br + 2, "wide", 10, cplx=True)
        C1 = make_mat(600 + trial, m, n, m + 2, "u", cplx=True, pad=0.125)
        C2 = C1.copy(order="F")
        al, be = complex(0.5, -1.25), complex(-0.75, 0.25)
        st_o = oracle.zgemm(ta, tb, m, n, k, al, A, Ar + 1, B, Br + 2, be, C1, m + 2, s)
        st_r = ref.zgemm(ta, tb, m, n, k, al, A, Ar + 1, B, Br + 2, be, C2, m + 2, s)
        assert st_o == st_r == 0, (ta, tb, m, n, k, s)
        assert np.array_equal(bits(C1), bits(C2)), (ta, tb, m, n, k, s)


@pytest.mark.parametrize("k,s", [(1500, 12), (2100, 17), (3000, 20), (700, 24)])
def test_long_k_oracle_against_reference_build(oracle, ref, k, s):
    """longer k with wide exponent ranges: tk on both sides of the narrow / wide boundary (62)"""
    m, n = 33, 29
    A = make_mat(700 + k, m, k, m + 3, "wide", 30)
    B = make_mat(800 + k, k, n, k + 1, "wide", 30)
    C1 = make_mat(900 + k, m, n, m, "u")
    C2 = C1.copy(order="F")
    st_o = oracle.dgemm("N", "N", m, n, k, 1.0, A, m + 3, B, k + 1, 0.5, C1, m, s)
    st_r, _ = ref.dgemm("N", "N", m, n, k, 1.0, A, m + 3, B, k + 1, 0.5, C2, m, s)
    assert st_o == st_r == 0
    assert np.array_equal(bits(C1), bits(C2)), oracle.plan(s, k).tk


def test_reference_own_suite_passes():
    """the reference's tests/test_ozaki2.cpp, built for the host, passes its quick suite"""
    exe = os.path.join(ROOT, "oracle", "_ref", "test_ozaki2")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/test_ozaki2 is not present")
    r = subprocess.run([exe, "--quick"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    assert ", 0 failed" in r.stdout
