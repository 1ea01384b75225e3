"""Generates the golden fixtures of tests/golden/ from the reference itself.

The reference (MacraMacra/OS2-Xe, src/ozaki2_gpu.hpp) is compiled for the host against the CPU
SYCL/oneMKL stand-in by `make -C oracle ref`; this script drives that build through
oracle/pyoracle.Ref and stores inputs and outputs:

  plans.json        make_plan(s, k) for s = 2..24 and several k: tk, NL, M, W_t, y_t
  split_*.npz       launch_split residues (the reference's unit_split inputs: U(-1,1),
                    U * 2^-[0,120), zeros / -0 / subnormals; narrow and wide paths)
  crt_*.npz         launch_crt on exact integers |x| <= M/4 given as unreduced int32 residues
  dgemm_cases.npz   Ozaki2::gemm end to end on small cases (all op pairs, alpha/beta, ld pads)
  zgemm_cases.npz   Ozaki2::zgemm end to end (all nine op pairs, complex alpha/beta)

Run from the repository root: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from common import make_mat, op_shape  # noqa: E402
from pyoracle import Ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PLAN_KS = [1, 16, 129, 1024, 2000, 8192, 131071, 262144, 1000000]
SPLIT_CASES = [(8, 24), (12, 40), (16, 55), (18, 62), (20, 70), (24, 85), (24, 100)]


def make_plans(ref):
    out = []
    for s in range(2, 25):
        for k in PLAN_KS:
            try:
                p = ref.plan(s, k)
            except ValueError:
                out.append({"s": s, "k": k, "invalid": True})
                continue
            out.append({"s": s, "k": k, "tk": p["tk"], "nl": p["nl"], "log2M": p["log2M"], "m": p["m"],
                        "y": p["y"], "M": hex(p["M"]), "W": [hex(w) for w in p["W"]]})
    mfb = {f"{k}:{b}": ref.moduli_for_bits(k, b) for k in [1, 16, 1024, 2000, 8192, 131071, 300000]
           for b in [1, 20, 40, 53, 60, 80, 90, 101]}
    with open(os.path.join(OUT, "plans.json"), "w") as f:
        json.dump({"plans": out, "moduli_for_bits": mfb}, f, indent=0)


def make_split(ref):
    rng = np.random.default_rng(1234)
    rows = 512
    for s, tk in SPLIT_CASES:
        X = np.zeros((rows, 3))
        X[:, 0] = rng.uniform(-1, 1, rows)
        X[:, 1] = rng.uniform(-1, 1, rows) * np.ldexp(1.0, -rng.integers(0, 120, rows))
        X[:, 2] = rng.uniform(-1, 1, rows) * np.ldexp(1.0, -1030 - rng.integers(0, 40, rows))
        X[0::7, 2] = 0.0
        X[1::7, 2] = -0.0
        ex = np.array([tk - np.frexp(np.abs(X[:, c]).max())[1] for c in range(3)], np.int32)
        P = ref.split(s, tk, X, ex, per_row=False)
        np.savez_compressed(os.path.join(OUT, f"split_s{s}_tk{tk}.npz"), X=X, ex=ex, P=P, s=s, tk=tk)


def make_crt(ref):
    rng = np.random.default_rng(777)
    n = 256
    data = {}
    for s in range(2, 25):
        p = ref.plan(s, 16)
        M = p["M"]
        Mq = M // 4
        xs = []
        for i in range(n):
            bits = Mq.bit_length() if i < 16 else int(rng.integers(0, Mq.bit_length() + 1))
            x = int.from_bytes(rng.bytes(32), "little") & ((1 << bits) - 1)
            x = Mq if i < 8 else min(x, Mq)
            if i == 8:
                x = 0
            if i != 8 and rng.integers(0, 2):
                x = -x
            xs.append(x)
        D = rng.integers(-20, 21, n).astype(np.int32)
        E = np.array([3], np.int32)
        Ct = np.zeros((s, n), np.int64)
        for i, x in enumerate(xs):
            for t in range(s):
                m = p["m"][t]
                Ct[t, i] = (x % m) + int(rng.integers(-10 ** 6, 10 ** 6 + 1)) * m
        out = ref.crt(s, Ct.astype(np.int32), n, 1, D, E)
        data[f"Ct{s}"] = Ct.astype(np.int32)
        data[f"D{s}"] = D
        data[f"out{s}"] = out
    np.savez_compressed(os.path.join(OUT, "crt_cases.npz"), **data)


# ta, tb, m, n, k, s, alpha, beta, kind, width, ld_extra, ldc_extra, seed. Inputs come from
# tests/common.make_mat(seed, ...), so the fixtures keep only the reference's outputs.
DGEMM_CASES = [
    *[(ta, tb, 1, 1, 1, 8, 1.0, 0.0, "h", 0, 0, 0, 11) for ta in "NT" for tb in "NT"],
    *[(ta, tb, 37, 53, 129, 12, 1.0, 0.0, "wide", 6, 3, 5, 12) for ta in "NT" for tb in "NT"],
    *[(ta, tb, 130, 7, 1, 6, 1.0, 0.0, "wide", 10, 0, 0, 13) for ta in "NT" for tb in "NT"],
    *[(ta, tb, 77, 65, 300, 14, -1.5, 0.25, "h", 0, 0, 2, 14) for ta in "NT" for tb in "NT"],
    ("N", "N", 64, 48, 1000, 12, 1.0, 0.0, "int", 0, 0, 0, 15),
    ("T", "T", 63, 31, 777, 14, 1.0, 0.0, "int", 0, 1, 1, 16),
    ("N", "N", 40, 40, 2048, 16, 1.0, 0.0, "maxmag", 0, 0, 0, 17),
    ("N", "N", 40, 40, 2048, 24, 1.0, 0.0, "maxmag", 0, 0, 0, 18),
    ("N", "T", 96, 80, 513, 20, 1.0, 0.0, "wide", 20, 0, 0, 19),
    ("T", "N", 33, 65, 1025, 16, 1.5, -0.5, "u", 0, 0, 16, 20),
    ("N", "N", 160, 140, 200, 10, 1.0, 0.0, "wide", 4, 0, 0, 21),
]
# ta, tb, m, n, k, s, alpha, beta, kind, width, ld_extra, seed
ZGEMM_CASES = [
    *[(ta, tb, 37, 29, 101, 14, 1 + 0j, 0j, "wide", 6, 3, 31) for ta in "NTC" for tb in "NTC"],
    ("N", "C", 64, 48, 300, 16, 0.5 - 1.25j, 0.25 + 2j, "u", 0, 1, 32),
    ("C", "N", 40, 36, 260, 16, 1 + 0.5j, 0.25 - 1j, "u", 0, 8, 33),
    ("N", "T", 60, 70, 900, 14, 1 + 0j, 0j, "int", 0, 0, 34),
    ("C", "N", 32, 32, 700, 24, 1 + 0j, 0j, "maxmag", 0, 0, 35),
]


def dgemm_inputs(case):
    ta, tb, m, n, k, s, al, be, kind, width, ldx, ldcx, seed = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(seed, Ar, Ac, Ar + ldx, kind, width)
    B = make_mat(seed + 1000, Br, Bc, Br + ldx, kind, width)
    C0 = make_mat(seed + 2000, m, n, m + ldcx, "u", pad=0.125)
    return A, B, C0


def zgemm_inputs(case):
    ta, tb, m, n, k, s, al, be, kind, width, ldx, seed = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(seed, Ar, Ac, Ar + ldx, kind, width, cplx=True)
    B = make_mat(seed + 1000, Br, Bc, Br + ldx, kind, width, cplx=True)
    C0 = make_mat(seed + 2000, m, n, m + ldx, "u", cplx=True, pad=0.125)
    return A, B, C0


def make_gemm(ref):
    data = {}
    for ci, case in enumerate(DGEMM_CASES):
        ta, tb, m, n, k, s, al, be = case[:8]
        A, B, C0 = dgemm_inputs(case)
        Cr = C0.copy(order="F")
        st, _ = ref.dgemm(ta, tb, m, n, k, al, A, A.shape[0], B, B.shape[0], be, Cr, Cr.shape[0], s)
        assert st == 0
        data[f"C{ci}"] = Cr
    np.savez_compressed(os.path.join(OUT, "dgemm_cases.npz"), meta=json.dumps([list(c) for c in DGEMM_CASES]),
                        **data)
    data = {}
    for ci, case in enumerate(ZGEMM_CASES):
        ta, tb, m, n, k, s, al, be = case[:8]
        A, B, C0 = zgemm_inputs(case)
        Cr = C0.copy(order="F")
        assert ref.zgemm(ta, tb, m, n, k, al, A, A.shape[0], B, B.shape[0], be, Cr, Cr.shape[0], s) == 0
        data[f"C{ci}"] = Cr
    meta = [list(c[:6]) + [[c[6].real, c[6].imag], [c[7].real, c[7].imag]] + list(c[8:]) for c in ZGEMM_CASES]
    np.savez_compressed(os.path.join(OUT, "zgemm_cases.npz"), meta=json.dumps(meta), **data)


if __name__ == "__main__":
    ref = Ref()
    ref.set_threads(os.cpu_count() or 1)
    make_plans(ref)
    make_split(ref)
    make_crt(ref)
    make_gemm(ref)
    print("golden fixtures written to", OUT)
