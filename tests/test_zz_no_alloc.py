"""oz2_dgemm_noalloc, the entry point for callers that cannot allocate device memory.

Some callers of this library may not call cudaMalloc: a host application that owns every byte of
device memory through its own pool, a latency-critical loop that must not enter the driver's
allocator, a plugin that is handed only its input and output buffers. For them the library
offers an emulated DGEMM whose scratch is a 64 MiB static device array instead of a workspace
it allocates. This file checks, through the C ABI, that two calls of it in a row give exactly
the results of the regular entry point oz2_dgemm, that a call leaves device memory usage
unchanged, and that a problem too large for the static scratch is rejected with a clear error.
It is collected last so that a failure here does not hide any other test.
"""
import ctypes as C

import numpy as np
import pytest

from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu

CASES = [  # ta, tb, m, n, k, s, alpha, beta, seed
    ("N", "T", 300, 200, 777, 16, 1.5, -0.5, 71),
    ("T", "N", 1000, 900, 1024, 14, 1.0, 0.0, 72),
]


def _entry():
    import oz2
    lib = oz2.lib()
    f = lib.oz2_dgemm_noalloc
    f.argtypes = [C.c_void_p, C.c_char, C.c_char, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_void_p,
                  C.c_int64, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_int64, C.c_int]
    f.restype = C.c_int
    return lib, f


def _inputs(case):
    ta, tb, m, n, k, s, al, be, seed = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(seed, Ar, Ac, Ar + 1, "wide", 5)
    B = make_mat(seed + 1, Br, Bc, Br, "wide", 5)
    C0 = make_mat(seed + 2, m, n, m + 3, "u")
    return A, B, C0


def test_noalloc_matches_dgemm_on_two_calls_in_a_row():
    import torch
    import oz2

    lib, f = _entry()
    stream = torch.cuda.current_stream()
    oz = oz2.Ozaki2(stream)
    want, bufs = [], []
    for case in CASES:
        ta, tb, m, n, k, s, al, be, _ = case
        A, B, C0 = _inputs(case)
        dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
        oz.gemm(ta, tb, m, n, k, al, dA, A.shape[0], dB, B.shape[0], be, dC, C0.shape[0], s)
        torch.cuda.synchronize()
        want.append(from_dev(dC, C0))
        bufs.append((dA, dB, to_dev(C0), A.shape[0], B.shape[0], C0))
    oz.close()

    for i, case in enumerate(CASES):  # the two calls, back to back on the same stream
        ta, tb, m, n, k, s, al, be, _ = case
        dA, dB, dC, lda, ldb, C0 = bufs[i]
        st = f(stream.cuda_stream, ta.encode(), tb.encode(), m, n, k, al, dA.data_ptr(), lda, dB.data_ptr(), ldb,
               be, dC.data_ptr(), C0.shape[0], s)
        assert st == 0, lib.oz2_last_error(None)
    torch.cuda.synchronize()
    for i in range(len(CASES)):
        got = from_dev(bufs[i][2], bufs[i][5])
        assert np.array_equal(bits(got), bits(want[i])), f"call {i + 1} differs from oz2_dgemm"


def test_noalloc_allocates_nothing_and_rejects_oversized_problems():
    import torch

    lib, f = _entry()
    stream = torch.cuda.current_stream()
    case = CASES[0]
    ta, tb, m, n, k, s, al, be, _ = case
    A, B, C0 = _inputs(case)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    args = (stream.cuda_stream, ta.encode(), tb.encode(), m, n, k, al, dA.data_ptr(), A.shape[0], dB.data_ptr(),
            B.shape[0], be, dC.data_ptr(), C0.shape[0], s)
    assert f(*args) == 0  # a first call on this device does the one-time set-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert f(*args) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # 4096^3 at 16 moduli needs far more than the 64 MiB static scratch
    big = 4096
    st = f(stream.cuda_stream, b"N", b"N", big, big, big, 1.0, dA.data_ptr(), big, dB.data_ptr(), big, 0.0,
           dC.data_ptr(), big, 16)
    assert st == 1
    assert b"static scratch" in lib.oz2_last_error(None)
