"""Grouped calls with adaptive problems (num_moduli = -1) beside fixed-s ones.

A grouped problem whose num_moduli is S_ADAPTIVE takes the adaptive s per tile (mode 0 with the
shipped model, 53-bit target). The fixed-s problems of the same call must equal plain gemm()
calls bit for bit, the adaptive ones must equal a separate gemm_adaptive call on the same
problems bit for bit and lie within the DGEMM-level bound; graph mode and other negative s are
rejected before anything runs.
"""
import numpy as np
import pytest

from common import bits, from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def gz():
    import torch
    import oz2
    h = oz2.Ozaki2(torch.cuda.current_stream())
    h.load_model()
    yield h
    h.close()


def wide(seed, rows, cols, phi, offsets):
    rng = np.random.default_rng(seed)
    X = (rng.random((rows, cols)) - 0.5) * np.exp(phi * rng.standard_normal((rows, cols)))
    X = X * np.ldexp(1.0, rng.integers(-offsets, offsets + 1, (rows, 1)))
    return np.asfortranarray(X)


SPECS = [  # m, n, k, phi, s (-1: adaptive)
    (300, 200, 500, 1.0, 16),
    (700, 600, 900, 3.0, -1),
    (129, 257, 1500, 0.5, 12),
    (520, 530, 640, 6.0, -1),
    (64, 900, 300, 2.0, 20),
    (1030, 257, 2000, 8.0, -1),
]


def make(i, m, n, k, phi):
    A = wide(10 + i, m, k, phi, 30)
    B = np.asfortranarray(wide(20 + i, n, k, phi, 30).T)
    C0 = np.asfortranarray(np.random.default_rng(30 + i).random((m, n)))
    return A, B, C0


def dd_ratio(h, m, n, k, dA, dB, dC):
    import torch
    hi = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    h.dd_reference(m, n, k, dA, m, dB, k, hi, lo, ab)
    return h.error_ratio(m, n, k, dC, m, hi, lo, ab, 53)


def test_mixed_grouped_call(gz):
    import torch
    import oz2
    data = [make(i, m, n, k, phi) for i, (m, n, k, phi, s) in enumerate(SPECS)]
    dev = [(to_dev(A), to_dev(B), to_dev(C0)) for A, B, C0 in data]
    probs = [("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, s)
             for (m, n, k, phi, s), (dA, dB, dC) in zip(SPECS, dev)]
    gz.gemm_grouped(probs)
    torch.cuda.synchronize()
    gz.check_device_error()
    mixed = [from_dev(dC, C0) for (_, _, dC), (_, _, C0) in zip(dev, data)]

    # the fixed-s problems against plain calls
    for i, (m, n, k, phi, s) in enumerate(SPECS):
        if s == oz2.S_ADAPTIVE:
            continue
        dA, dB, _ = dev[i]
        dC = to_dev(data[i][2])
        gz.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, s)
        torch.cuda.synchronize()
        assert np.array_equal(bits(from_dev(dC, data[i][2])), bits(mixed[i])), SPECS[i]

    # the adaptive problems against one gemm_adaptive call on them alone, and the bound
    ad = [i for i, sp in enumerate(SPECS) if sp[4] == oz2.S_ADAPTIVE]
    dCs = {i: to_dev(data[i][2]) for i in ad}
    gz.gemm_adaptive([("N", "N", SPECS[i][0], SPECS[i][1], SPECS[i][2], 1.0, dev[i][0], SPECS[i][0], dev[i][1],
                       SPECS[i][2], 0.0, dCs[i], SPECS[i][0], 16) for i in ad], 53, gz.ADAPTIVE_MLP)
    torch.cuda.synchronize()
    gz.check_device_error()
    for i in ad:
        m, n, k = SPECS[i][:3]
        assert np.array_equal(bits(from_dev(dCs[i], data[i][2])), bits(mixed[i])), SPECS[i]
        assert dd_ratio(gz, m, n, k, dev[i][0], dev[i][1], dev[i][2]) <= 1.0, SPECS[i]


def test_rejections(gz):
    import torch
    import oz2
    m = n = k = 64
    A, B, C0 = make(0, m, n, k, 1.0)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C0)
    with pytest.raises(ValueError):
        gz.gemm_grouped([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, -2)])
    gz.set_graph_mode(True)
    try:
        with pytest.raises(ValueError, match="graph mode"):
            gz.gemm_grouped([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, oz2.S_ADAPTIVE)])
    finally:
        gz.set_graph_mode(False)
    torch.cuda.synchronize()
    assert np.array_equal(bits(from_dev(dC, C0)), bits(C0))  # nothing ran
