"""ctypes bindings for the two CPU checkers of the Ozaki-II path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs, never by the product package.

- ``Oracle``: oracle/liboz2_oracle.so, the C restatement of the reference arithmetic.
- ``Ref``:    oracle/_ref/libozref.so, MacraMacra/OS2-Xe's own header compiled for the host
              against the CPU SYCL/oneMKL stand-in (present only where it was built).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboz2_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libozref.so")

_i64, _i32, _dbl, _vp, _chr = C.c_int64, C.c_int, C.c_double, C.c_void_p, C.c_char
NON_FINITE = -(2 ** 31)


def _ptr(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def _op(c):
    return c.encode() if isinstance(c, str) else c


class Plan(C.Structure):
    _fields_ = [("s", _i32), ("nl", _i32), ("tk", _i32), ("log2M", _dbl),
                ("m", C.c_uint32 * 32), ("y", C.c_uint32 * 32),
                ("W", (C.c_uint32 * 8) * 32), ("M", C.c_uint32 * 8)]

    def big(self, words):
        return sum(int(w) << (32 * i) for i, w in enumerate(words))

    @property
    def Mint(self):
        return self.big(self.M)

    def Wint(self, t):
        return self.big(self.W[t])


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle)")
        L = self.lib = C.CDLL(path)
        L.oz2o_make_plan.argtypes = [_i32, _i64, C.POINTER(Plan)]
        L.oz2o_make_plan_ext.argtypes = [_i32, _i64, C.POINTER(Plan)]
        L.oz2o_precision_bits.argtypes = [_i64, _i32, C.POINTER(_i32)]
        L.oz2o_moduli_for_bits.argtypes = [_i64, _i32]
        L.oz2o_exponent.argtypes = [C.c_uint64, _i32]
        L.oz2o_residue.argtypes = [_dbl, _i32, C.c_uint32]
        L.oz2o_residue.restype = C.c_int8
        L.oz2o_split.argtypes = [_vp, _i64, _i64, _i64, _vp, _i32, C.POINTER(Plan), _vp, _i64, _i64]
        L.oz2o_crt.argtypes = [C.POINTER(Plan), _vp, _i32]
        L.oz2o_crt.restype = _dbl
        gemm_args = [_chr, _chr, _i64, _i64, _i64]
        L.oz2o_dgemm.argtypes = gemm_args + [_dbl, _vp, _i64, _vp, _i64, _dbl, _vp, _i64, _i32]
        L.oz2o_dgemm_ext.argtypes = gemm_args + [_dbl, _vp, _i64, _vp, _i64, _dbl, _vp, _i64, _i32]
        L.oz2o_zgemm.argtypes = gemm_args + [_vp, _vp, _i64, _vp, _i64, _vp, _vp, _i64, _i32]
        L.oz2o_exponents.argtypes = gemm_args + [_vp, _i64, _vp, _i64, _i32, _i32, _vp, _vp]
        L.oz2o_dd_gemm.argtypes = gemm_args + [_vp, _i64, _vp, _i64, _vp, _vp]
        L.oz2o_dd_zgemm.argtypes = gemm_args + [_vp, _i64, _vp, _i64, _vp, _vp]
        L.oz2o_bound_ratio.argtypes = gemm_args + [_i32, _vp, _i64, _vp, _i64, _dbl, _dbl, _vp, _vp, _i64, _vp, _vp]
        L.oz2o_bound_ratio.restype = _dbl
        L.oz2o_zbound_ratio.argtypes = gemm_args + [_i32, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _vp]
        L.oz2o_zbound_ratio.restype = _dbl
        L.oz2o_metrics.argtypes = [_i64, _vp, _vp, _vp, _vp, _vp]
        L.oz2o_set_threads.argtypes = [_i32]
        L.oz1o_dgemm.argtypes = [_i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i32]

    def set_threads(self, n):
        self.lib.oz2o_set_threads(n)

    def ozaki1(self, m, n, k, A, lda, B, ldb, C_, ldc, L):
        """Ozaki-I restatement: C = A B (N, N), column-major; returns the status"""
        return self.lib.oz1o_dgemm(m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(C_), ldc, L)

    def plan(self, s, k):
        p = Plan()
        st = self.lib.oz2o_make_plan(s, k, C.byref(p))
        if st:
            raise ValueError(f"oracle plan(s={s}, k={k}) status {st}")
        return p

    def plan_ext(self, s, k):
        """the plan for s in [2, 32]: the reference's up to 24, the library's extended sets above"""
        p = Plan()
        st = self.lib.oz2o_make_plan_ext(s, k, C.byref(p))
        if st:
            raise ValueError(f"oracle plan_ext(s={s}, k={k}) status {st}")
        return p

    def precision_bits(self, k, s):
        out = _i32()
        st = self.lib.oz2o_precision_bits(k, s, C.byref(out))
        if st:
            raise ValueError(f"s={s} too small for k={k}")
        return out.value

    def moduli_for_bits(self, k, bits):
        return self.lib.oz2o_moduli_for_bits(k, bits)

    def exponent(self, maxbits, tk):
        return self.lib.oz2o_exponent(maxbits, tk)

    def split(self, X, ex, per_row, plan):
        """X: (rows, cols) column-major float64 (Fortran order). Returns int8 (s, cols, rows)."""
        X = np.asfortranarray(X, dtype=np.float64)
        rows, cols = X.shape
        P = np.zeros((plan.s, cols, rows), dtype=np.int8)
        ex = np.ascontiguousarray(ex, dtype=np.int32)
        self.lib.oz2o_split(_ptr(X), rows, rows, cols, _ptr(ex), int(per_row), C.byref(plan), _ptr(P), rows,
                            rows * cols)
        return P

    def crt(self, plan, residues, shift):
        r = np.ascontiguousarray(residues, dtype=np.int64)
        return self.lib.oz2o_crt(C.byref(plan), _ptr(r), shift)

    def dgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, s):
        return self.lib.oz2o_dgemm(_op(ta), _op(tb), m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C_),
                                   ldc, s)

    def dgemm_ext(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, s):
        return self.lib.oz2o_dgemm_ext(_op(ta), _op(tb), m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C_),
                                   ldc, s)

    def zgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, s):
        al = np.array([alpha.real, alpha.imag])
        be = np.array([beta.real, beta.imag])
        return self.lib.oz2o_zgemm(_op(ta), _op(tb), m, n, k, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be),
                                   _ptr(C_), ldc, s)

    def exponents(self, ta, tb, m, n, k, A, lda, B, ldb, tk, cplx=False):
        D = np.zeros(m, np.int32)
        E = np.zeros(n, np.int32)
        self.lib.oz2o_exponents(_op(ta), _op(tb), m, n, k, _ptr(A), lda, _ptr(B), ldb, tk, int(cplx), _ptr(D),
                                _ptr(E))
        return D, E

    def dd_gemm(self, ta, tb, m, n, k, A, lda, B, ldb):
        hi = np.zeros(m * n)
        lo = np.zeros(m * n)
        self.lib.oz2o_dd_gemm(_op(ta), _op(tb), m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(hi), _ptr(lo))
        return hi, lo

    def dd_zgemm(self, ta, tb, m, n, k, A, lda, B, ldb):
        hi = np.zeros(2 * m * n)
        lo = np.zeros(2 * m * n)
        self.lib.oz2o_dd_zgemm(_op(ta), _op(tb), m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(hi), _ptr(lo))
        return hi, lo

    def bound_ratio(self, ta, tb, m, n, k, s, A, lda, B, ldb, alpha, beta, C0, C_, ldc, hi, lo):
        return self.lib.oz2o_bound_ratio(_op(ta), _op(tb), m, n, k, s, _ptr(A), lda, _ptr(B), ldb, alpha, beta,
                                         _ptr(C0), _ptr(C_), ldc, _ptr(hi), _ptr(lo))

    def zbound_ratio(self, ta, tb, m, n, k, s, A, lda, B, ldb, alpha, beta, C0, C_, ldc, hi, lo):
        al = np.array([alpha.real, alpha.imag])
        be = np.array([beta.real, beta.imag])
        return self.lib.oz2o_zbound_ratio(_op(ta), _op(tb), m, n, k, s, _ptr(A), lda, _ptr(B), ldb, _ptr(al),
                                          _ptr(be), _ptr(C0), _ptr(C_), ldc, _ptr(hi), _ptr(lo))

    def metrics(self, C_, hi, lo, absAB=None):
        out = np.zeros(5)
        C_ = np.ascontiguousarray(C_, dtype=np.float64)
        self.lib.oz2o_metrics(C_.size, _ptr(C_), _ptr(hi), _ptr(lo), _ptr(absAB), _ptr(out))
        return dict(zip(["ulp_max", "ulp_mean", "cr_frac", "ab_max", "fro_rel"], out.tolist()))


class Ref:
    """The reference itself (src/ozaki2_gpu.hpp) built for the host; see oracle/ref_driver.cpp."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle ref)")
        L = self.lib = C.CDLL(path)
        L.ozref_make_plan.argtypes = [_i32, _i64, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_dbl), _vp, _vp, _vp,
                                      _vp]
        L.ozref_precision_bits.argtypes = [_i64, _i32, C.POINTER(_i32)]
        L.ozref_moduli_for_bits.argtypes = [_i64, _i32]
        L.ozref_split.argtypes = [_i32, _i32, _vp, _i64, _i64, _vp, _i32, _vp]
        L.ozref_crt.argtypes = [_i32, _vp, _i64, _i64, _vp, _vp, _dbl, _dbl, _vp, _i64]
        gemm_args = [_chr, _chr, _i64, _i64, _i64]
        L.ozref_dgemm.argtypes = gemm_args + [_dbl, _vp, _i64, _vp, _i64, _dbl, _vp, _i64, _i32, C.c_size_t, _vp]
        L.ozref_zgemm.argtypes = gemm_args + [_vp, _vp, _i64, _vp, _i64, _vp, _vp, _i64, _i32, C.c_size_t]
        L.ozref_set_threads.argtypes = [_i32]
        L.ozref_ozaki1.argtypes = [_i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i32]

    def set_threads(self, n):
        self.lib.ozref_set_threads(n)

    def ozaki1(self, m, n, k, A, lda, B, ldb, C_, ldc, L):
        """the reference's oz1::Ozaki1::gemm: C = A B (N, N); returns the status"""
        return self.lib.ozref_ozaki1(m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(C_), ldc, L)

    def plan(self, s, k):
        tk, nl, l2 = _i32(), _i32(), _dbl()
        m = np.zeros(24, np.uint32)
        y = np.zeros(24, np.uint32)
        W = np.zeros((24, 8), np.uint32)
        M = np.zeros(8, np.uint32)
        st = self.lib.ozref_make_plan(s, k, C.byref(tk), C.byref(nl), C.byref(l2), _ptr(m), _ptr(y), _ptr(W),
                                      _ptr(M))
        if st:
            raise ValueError(f"reference plan(s={s}, k={k}) status {st}")
        big = lambda ws: sum(int(w) << (32 * i) for i, w in enumerate(ws))
        return dict(tk=tk.value, nl=nl.value, log2M=l2.value, m=m[:s].tolist(), y=y[:s].tolist(),
                    W=[big(W[t]) for t in range(s)], M=big(M))

    def precision_bits(self, k, s):
        out = _i32()
        st = self.lib.ozref_precision_bits(k, s, C.byref(out))
        if st:
            raise ValueError(f"s={s} too small for k={k}")
        return out.value

    def moduli_for_bits(self, k, bits):
        return self.lib.ozref_moduli_for_bits(k, bits)

    def split(self, s, tk, X, ex, per_row):
        """X (rows, cols) with rows % 4 == 0; returns int8 (s, cols, rows)."""
        X = np.asfortranarray(X, dtype=np.float64)
        rows, cols = X.shape
        assert rows % 4 == 0
        P = np.zeros((s, cols, rows), np.int8)
        ex = np.ascontiguousarray(ex, dtype=np.int32)
        st = self.lib.ozref_split(s, tk, _ptr(X), rows, cols, _ptr(ex), int(per_row), _ptr(P))
        assert st == 0
        return P

    def crt(self, s, Ct, mb, nb, D, E, alpha=1.0, beta=0.0, C_=None):
        Ct = np.ascontiguousarray(Ct, dtype=np.int32)
        if C_ is None:
            C_ = np.zeros(mb * nb)
        st = self.lib.ozref_crt(s, _ptr(Ct), mb, nb, _ptr(np.ascontiguousarray(D, np.int32)),
                                _ptr(np.ascontiguousarray(E, np.int32)), alpha, beta, _ptr(C_), mb)
        assert st == 0
        return C_

    def dgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, s, ws_limit=0):
        tiling = np.zeros(6, np.int64)
        st = self.lib.ozref_dgemm(_op(ta), _op(tb), m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C_), ldc,
                                  s, ws_limit, _ptr(tiling))
        return st, tiling

    def zgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, s, ws_limit=0):
        al = np.array([alpha.real, alpha.imag])
        be = np.array([beta.real, beta.imag])
        return self.lib.ozref_zgemm(_op(ta), _op(tb), m, n, k, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be),
                                    _ptr(C_), ldc, s, ws_limit)


def ref_available():
    return os.path.exists(REF_SO)
