"""oz2_dgemm_noalloc, the entry point for callers that cannot allocate device memory.

Some callers of this library may not call cudaMalloc: a host application that owns every byte of
device memory through its own pool, a latency-critical loop that must not enter the driver's
allocator, a plugin that is handed only its input and output buffers. For them the library
offers an emulated DGEMM whose scratch is a 64 MiB static device array instead of a workspace
it allocates. This file checks, through the C ABI, that two calls of it in a row give exactly
the results of the regular entry point oz2_dgemm and of the oracle; that it works in a fresh
process that never created a handle (the process such a caller runs in); that a call leaves
device memory usage unchanged; that the early returns (k = 0, alpha = 0), beta = 0 over a C full
of NaN and op 'C' behave like oz2_dgemm; that the largest problem the static scratch holds runs
and one just past it is rejected with a clear error; and that a GEMM whose bounded waits run out
is reported by oz2_noalloc_check_device_error. It is collected last so that a failure here does
not hide any other test.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from common import ROOT, bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu

SCRATCH = 64 << 20  # the static scratch of oz2_dgemm_noalloc, bytes

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
    lib.oz2_noalloc_check_device_error.argtypes = [C.c_void_p]
    lib.oz2_noalloc_check_device_error.restype = C.c_int
    return lib, f


def _inputs(case):
    ta, tb, m, n, k, s, al, be, seed = case
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(seed, Ar, Ac, Ar + 1, "wide", 5)
    B = make_mat(seed + 1, Br, Bc, Br, "wide", 5)
    C0 = make_mat(seed + 2, m, n, m + 3, "u")
    return A, B, C0


def _oracle_c(oracle, case, A, B, C0):
    ta, tb, m, n, k, s, al, be, _ = case
    Co = C0.copy(order="F")
    assert oracle.dgemm(ta, tb, m, n, k, al, A, max(A.shape[0], 1), B, max(B.shape[0], 1), be, Co, C0.shape[0],
                        s) == 0
    return Co


def _scratch_need(m, n, k, s):
    """bytes of static scratch a call uses: error word, row / column maxima, the INT8 planes of
    both operands (rows padded to 256 and 128, k to 128), the residues (rows padded to 32) and
    8 KiB of item tables, each region 256-byte aligned"""
    a = lambda v: (v + 255) // 256 * 256  # noqa: E731
    kp = -(-k // 128) * 128
    o = a(a(256 + 8 * m) + 8 * n)
    o = a(o + s * (-(-m // 256) * 256) * kp)
    o = a(o + s * (-(-n // 128) * 128) * kp)
    return a(o + s * n * (-(-m // 32) * 32)) + 8 * 1024


def test_noalloc_matches_dgemm_on_two_calls_in_a_row(oracle):
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
        got = from_dev(dC, C0)
        assert np.array_equal(bits(got), bits(_oracle_c(oracle, case, A, B, C0)))
        want.append(got)
        bufs.append((dA, dB, to_dev(C0), A.shape[0], B.shape[0], C0))
    oz.close()

    for i, case in enumerate(CASES):  # the two calls, back to back on the same stream
        ta, tb, m, n, k, s, al, be, _ = case
        dA, dB, dC, lda, ldb, C0 = bufs[i]
        st = f(stream.cuda_stream, ta.encode(), tb.encode(), m, n, k, al, dA.data_ptr(), lda, dB.data_ptr(), ldb,
               be, dC.data_ptr(), C0.shape[0], s)
        assert st == 0, lib.oz2_last_error(None)
    assert lib.oz2_noalloc_check_device_error(stream.cuda_stream) == 0
    for i in range(len(CASES)):
        got = from_dev(bufs[i][2], bufs[i][5])
        assert np.array_equal(bits(got), bits(want[i])), f"call {i + 1} differs from oz2_dgemm"


CHILD = textwrap.dedent("""
    import ctypes as C, sys
    import numpy as np
    sys.path[:0] = {paths!r}
    import torch
    from common import from_dev, to_dev
    import oz2  # loads liboz2.so; creates no handle
    from test_zz_no_alloc import CASES, _entry, _inputs
    lib, f = _entry()
    st = torch.cuda.current_stream()
    outs = []
    for case in CASES:
        ta, tb, m, n, k, s, al, be, _ = case
        A, B, C0 = _inputs(case)
        dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
        rc = f(st.cuda_stream, ta.encode(), tb.encode(), m, n, k, al, dA.data_ptr(), A.shape[0], dB.data_ptr(),
               B.shape[0], be, dC.data_ptr(), C0.shape[0], s)
        assert rc == 0, lib.oz2_last_error(None)
        outs.append((dC, C0))
    assert lib.oz2_noalloc_check_device_error(st.cuda_stream) == 0, lib.oz2_last_error(None)
    np.savez({out!r}, *[from_dev(d, c0) for d, c0 in outs])
""")


def test_noalloc_in_a_fresh_process_without_a_handle(oracle, tmp_path):
    out = str(tmp_path / "noalloc.npz")
    paths = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "os2-xe_b200")]
    r = subprocess.run([sys.executable, "-c", CHILD.format(paths=paths, out=out)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.load(out)
    for i, case in enumerate(CASES):
        A, B, C0 = _inputs(case)
        assert np.array_equal(bits(got[f"arr_{i}"]), bits(_oracle_c(oracle, case, A, B, C0))), case


EDGE = [  # ta, tb, m, n, k, s, alpha, beta, seed; C0 kind
    (("N", "N", 130, 70, 0, 16, 1.5, -0.5, 81), "u"),     # k = 0: C = beta C
    (("N", "N", 130, 70, 300, 16, 0.0, 2.0, 82), "u"),    # alpha = 0: C = beta C
    (("T", "N", 130, 70, 300, 16, 1.0, 0.0, 83), "nan"),  # beta = 0 overwrites NaN
    (("C", "T", 200, 150, 640, 12, -0.75, 0.25, 84), "u"),  # 'C' equals 'T' for real data
]


@pytest.mark.parametrize("ci", range(len(EDGE)))
def test_noalloc_edge_cases_match_oracle(oracle, ci):
    import torch

    lib, f = _entry()
    case, kind = EDGE[ci]
    ta, tb, m, n, k, s, al, be, seed = case
    A, B, C0 = _inputs(case)
    if kind == "nan":
        C0[:m] = np.nan
    st = torch.cuda.current_stream()
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    rc = f(st.cuda_stream, ta.encode(), tb.encode(), m, n, k, al, dA.data_ptr(), max(A.shape[0], 1), dB.data_ptr(),
           max(B.shape[0], 1), be, dC.data_ptr(), C0.shape[0], s)
    assert rc == 0, lib.oz2_last_error(None)
    assert lib.oz2_noalloc_check_device_error(st.cuda_stream) == 0
    got = from_dev(dC, C0)
    assert np.array_equal(bits(got), bits(_oracle_c(oracle, case, A, B, C0))), case


def test_noalloc_allocates_nothing_and_takes_problems_up_to_its_scratch(oracle):
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

    # the largest k that fits at m = n = 256, s = 16, and the next k (one more 128-wide k block)
    mm = nn = 256
    kfit = max(kk for kk in range(128, 20000, 128) if _scratch_need(mm, nn, kk, 16) <= SCRATCH)
    assert _scratch_need(mm, nn, kfit + 1, 16) > SCRATCH
    cs = ("N", "N", mm, nn, kfit, 16, 1.0, 0.0, 91)
    A, B, C0 = _inputs(cs)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    rc = f(stream.cuda_stream, b"N", b"N", mm, nn, kfit, 1.0, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0],
           0.0, dC.data_ptr(), C0.shape[0], 16)
    assert rc == 0, lib.oz2_last_error(None)
    assert lib.oz2_noalloc_check_device_error(stream.cuda_stream) == 0
    assert np.array_equal(bits(from_dev(dC, C0)), bits(_oracle_c(oracle, cs, A, B, C0)))
    rc = f(stream.cuda_stream, b"N", b"N", mm, nn, kfit + 1, 1.0, dA.data_ptr(), A.shape[0], dB.data_ptr(),
           kfit + 1, 0.0, dC.data_ptr(), C0.shape[0], 16)
    assert rc == 1
    assert b"static scratch" in lib.oz2_last_error(None)
    # 4096^3 at 16 moduli needs far more than the 64 MiB static scratch
    big = 4096
    st = f(stream.cuda_stream, b"N", b"N", big, big, big, 1.0, dA.data_ptr(), big, dB.data_ptr(), big, 0.0,
           dC.data_ptr(), big, 16)
    assert st == 1
    assert b"static scratch" in lib.oz2_last_error(None)


def test_noalloc_reports_a_device_wait_that_ran_out(oracle):
    import torch
    import oz2

    lib, f = _entry()
    stream = torch.cuda.current_stream()
    case = CASES[1]
    ta, tb, m, n, k, s, al, be, _ = case
    A, B, C0 = _inputs(case)
    dA, dB = to_dev(A), to_dev(B)
    args = lambda dC: (stream.cuda_stream, ta.encode(), tb.encode(), m, n, k, al, dA.data_ptr(),  # noqa: E731
                       A.shape[0], dB.data_ptr(), B.shape[0], be, dC.data_ptr(), C0.shape[0], s)
    assert lib.oz2_noalloc_check_device_error(stream.cuda_stream) == 0
    try:
        oz2.set_failure_test(5_000_000, stall_mma=True)
        dC = to_dev(C0)
        assert f(*args(dC)) == 0
        assert lib.oz2_noalloc_check_device_error(stream.cuda_stream) == 4  # OZ2_ETIMEOUT
        assert b"ran out" in lib.oz2_last_error(None)
    finally:
        oz2.set_failure_test()
    assert lib.oz2_noalloc_check_device_error(stream.cuda_stream) == 0  # read and cleared
    dC = to_dev(C0)
    assert f(*args(dC)) == 0
    assert lib.oz2_noalloc_check_device_error(stream.cuda_stream) == 0
    assert np.array_equal(bits(from_dev(dC, C0)), bits(_oracle_c(oracle, case, A, B, C0)))
