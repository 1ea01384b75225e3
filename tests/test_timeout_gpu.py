"""The GEMM kernel's bounded waits, made to run out on purpose without faulting the GPU.

Every mbarrier wait of the persistent tcgen05 GEMM has a time limit (a kernel parameter). Here
the limit is cut to a few milliseconds and the MMA issuer is told to issue nothing: the
accumulator barrier the epilogue waits on and the ring slots the producer waits on are then never
released, exactly like a flag that nothing sets. The kernel must record a timeout code, drain
the copies it issued, free its tensor memory and return; the host must see OZ2_ETIMEOUT; and
the next ordinary call must be bit-exact again (the context is still usable).
"""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, to_dev

pytestmark = pytest.mark.gpu

WAIT_NS = 5_000_000  # 5 ms


def _case():
    m, n, k, s = 640, 384, 2048, 16
    A = make_mat(901, m, k, m, "u")
    B = make_mat(902, k, n, k, "u")
    C0 = make_mat(903, m, n, m, "u")
    return m, n, k, s, A, B, C0


def test_stalled_gemm_reports_timeout_and_the_next_call_is_exact(oz, oracle):
    import torch
    import oz2

    m, n, k, s, A, B, C0 = _case()
    want = C0.copy(order="F")
    assert oracle.dgemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.5, want, m, s) == 0
    dA, dB = to_dev(A), to_dev(B)
    oz.check_device_error()  # nothing pending before the test
    try:
        oz2.set_failure_test(WAIT_NS, stall_mma=True)
        dC = to_dev(C0)
        oz.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.5, dC, m, s)
        torch.cuda.synchronize()
    finally:
        oz2.set_failure_test()
    with pytest.raises(TimeoutError):
        oz.check_device_error()
    oz.check_device_error()  # the word was cleared by the read
    for _ in range(2):  # the same handle and stream compute normally again
        dC = to_dev(C0)
        oz.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.5, dC, m, s)
        torch.cuda.synchronize()
        oz.check_device_error()
        assert np.array_equal(bits(from_dev(dC, C0)), bits(want))


def test_failure_test_knob_rejects_negative_limits():
    import oz2
    with pytest.raises(ValueError):
        oz2.set_failure_test(-1)
