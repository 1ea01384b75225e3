"""Adaptive number of moduli per C tile: the MLP kernels against a torch fp32 restatement, the
tile features and analytic s against a numpy restatement of their definition, the probe (it
catches tiles run at too few moduli and passes tiles that meet the target), and the modes'
results: fixed s equals the plain product bit for bit, analytic s meets the DGEMM-level target
k 2^-53 (|A||B|)_ij against the double-double reference."""
import math

import numpy as np
import pytest

import adaptive_oracle
from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu

TILE = 512


@pytest.fixture(scope="module")
def az():
    """a handle of its own: these tests load MLP weights and change the adaptive options"""
    import torch
    import oz2
    h = oz2.Ozaki2(torch.cuda.current_stream())
    yield h
    h.close()


def info():
    import oz2
    return oz2.mlp_info()


def wide_rows(seed, rows, cols, phi, offsets):
    """(u - 0.5) exp(phi g) with per-row power-of-two offsets in [-offsets, offsets], column-major"""
    rng = np.random.default_rng(seed)
    X = (rng.random((rows, cols)) - 0.5) * np.exp(phi * rng.standard_normal((rows, cols)))
    if offsets:
        X = X * np.ldexp(1.0, rng.integers(-offsets, offsets + 1, (rows, 1)))
    return np.asfortranarray(X)


def const_class_params(cls):
    """an MLP whose softmax puts (nearly) all mass on one class: s = cls + 2 at any threshold"""
    i = info()
    P = [0.0] * i["params"]
    P[i["params"] - i["classes"] + cls] = 60.0
    return P


def torch_forward(params, feat):
    import torch
    i = info()
    F, H, Cn = i["features"], i["hidden"], i["classes"]
    P = torch.tensor(params, dtype=torch.float32, device=feat.device)
    o = 0
    W1 = P[o:o + H * F].view(H, F); o += H * F
    b1 = P[o:o + H]; o += H
    W2 = P[o:o + H * H].view(H, H); o += H * H
    b2 = P[o:o + H]; o += H
    W3 = P[o:o + Cn * H].view(Cn, H); o += Cn * H
    b3 = P[o:o + Cn]
    h1 = torch.relu(feat @ W1.T + b1)
    h2 = torch.relu(h1 @ W2.T + b2)
    return torch.softmax(h2 @ W3.T + b3, dim=1)


def test_mlp_inference_matches_torch_fp32(az):
    import torch
    from oz2 import adaptive
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    feat = torch.rand((1000, info()["features"]), generator=g, device="cuda")
    params = adaptive.init_params(seed=11)
    # larger biases so the decision is not always the first class
    params = [p * 3.0 for p in params]
    s, probs = az.mlp_infer(params, feat, 0.9, probs=True)
    want = torch_forward(params, feat)
    assert torch.allclose(probs, want, atol=2e-5, rtol=1e-4)
    cum = torch.cumsum(want, dim=1)
    ref_s = 2 + torch.clamp((cum < 0.9).sum(dim=1), max=info()["classes"] - 1)
    margin = (cum - 0.9).abs().min(dim=1).values
    clear = margin > 1e-4
    assert clear.float().mean() > 0.9
    assert torch.equal(s[clear].long(), ref_s[clear].long())
    assert int(s.min()) >= 2 and int(s.max()) <= 24


def test_mlp_training_fits_a_learnable_rule(az):
    import torch
    from oz2 import adaptive
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    feat = torch.rand((2048, info()["features"]), generator=g, device="cuda")
    labels = (2 + torch.floor(feat[:, 2] * 8) + torch.floor(feat[:, 0] * 8)).to(torch.int32)
    params, losses = az.mlp_train(feat, labels, adaptive.init_params(seed=1), epochs=150, lr=3e-3, seed=2)
    assert all(math.isfinite(x) for x in losses)
    assert losses[-1] < 0.5 * losses[0]
    s = az.mlp_infer(params, feat, 0.5)
    assert (s - labels).abs().le(1).float().mean().item() > 0.9


# the first list takes the fused scale + statistics pass (every k up to 16384), the second, with
# one longer k, the scale pass followed by the statistics pass
FEATURE_CASES = [[("N", "N", 700, 600, 300, 1.0, 10), ("T", "N", 513, 1030, 999, 4.0, 40),
                  ("N", "T", 128, 200, 5000, 0.0, 0), ("T", "T", 600, 520, 64, 8.0, 20)],
                 [("N", "N", 300, 130, 20000, 2.0, 30), ("T", "T", 90, 520, 700, 4.0, 10)]]


@pytest.mark.parametrize("case", range(len(FEATURE_CASES)))
def test_tile_features_and_analytic_s_match_host_restatement(oracle, az, case):
    import torch
    rng = np.random.default_rng(9)
    probs, dev = [], []
    for q, (ta, tb, m, n, k, phi, offs) in enumerate(FEATURE_CASES[case]):
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        A = wide_rows(100 + q, Ar, Ac, phi, offs)
        B = wide_rows(200 + q, Br, Bc, phi, offs)
        A[rng.random(A.shape) < 0.05] = 0.0  # zeros are counted apart
        if q == 0:
            A[3, :] = 0.0  # an all-zero row contributes nothing
        probs.append((ta, tb, m, n, k, A, B))
        C = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        dev.append((ta, tb, m, n, k, 1.0, to_dev(A), Ar, to_dev(B), Br, 0.0, C, m, 16))
    az.set_adaptive_options(TILE, 0.9)
    feat, s_an = az.tile_features(dev)
    want_f, want_s = adaptive_oracle.tile_features(oracle, probs)
    got_f = feat.cpu().numpy()
    assert got_f.shape == want_f.shape
    np.testing.assert_allclose(got_f[:, 0], want_f[:, 0], rtol=1e-6)
    assert np.array_equal(got_f[:, 1:], want_f[:, 1:])
    assert np.array_equal(s_an.cpu().numpy(), want_s)


def nn_problem(seed, m, n, k, phi, offsets):
    A = wide_rows(seed, m, k, phi, offsets)
    B = np.asfortranarray(wide_rows(seed + 1, n, k, phi, offsets).T)
    return A, B


def dd_check(az, m, n, k, dA, dB, dC, target_bits=53):
    import torch
    hi = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    az.dd_reference(m, n, k, dA, m, dB, k, hi, lo, ab)
    return az.error_ratio(m, n, k, dC, m, hi, lo, ab, target_bits)


def test_mode3_equals_plain_products(az):
    import torch
    probs, want = [], []
    for q, (ta, tb, m, n, k, s) in enumerate([("N", "T", 700, 530, 260, 14), ("T", "N", 300, 1100, 777, 18),
                                              ("T", "T", 1030, 90, 4100, 20)]):
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        A = make_mat(30 + q, Ar, Ac, Ar + 3, "wide", 8)
        B = make_mat(40 + q, Br, Bc, Br + 1, "wide", 8)
        C0 = make_mat(50 + q, m, n, m + 5, "u")
        p = (ta, tb, m, n, k, 1.25, to_dev(A), Ar + 3, to_dev(B), Br + 1, -0.5, to_dev(C0), m + 5, s)
        probs.append((p, C0))
        dC = to_dev(C0)
        az.gemm(*p[:11], dC, m + 5, s)
        want.append(from_dev(dC, C0))
    stats = az.gemm_adaptive([p for p, _ in probs], 53, az.ADAPTIVE_FIXED)
    torch.cuda.synchronize()
    for (p, C0), w in zip(probs, want):
        assert np.array_equal(bits(from_dev(p[11], C0)), bits(w))
    assert stats["tiles"] == sum(math.ceil(p[2] / TILE) * math.ceil(p[3] / TILE) for p, _ in probs)
    assert stats["sum_s"] == sum(p[13] * math.ceil(p[2] / TILE) * math.ceil(p[3] / TILE) for p, _ in probs)


@pytest.mark.parametrize("phi,offsets", [(0.0, 0), (1.0, 40), (4.0, 40), (8.0, 40)])
def test_analytic_modes_meet_the_target(az, phi, offsets):
    import torch
    m, n, k = 1100, 700, 1500
    A, B = nn_problem(int(phi * 10) + 7, m, n, k, phi, offsets)
    dA, dB = to_dev(A), to_dev(B)
    results = {}
    for mode in (az.ADAPTIVE_ANALYTIC_TILE, az.ADAPTIVE_ANALYTIC_PROBLEM):
        dC = torch.full((m * n,), 7.0, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, mode)
        ratio = dd_check(az, m, n, k, dA, dB, dC)
        results[mode] = (st, ratio)
        # tiles that 24 moduli do not bring to the target run as native FP64 GEMMs
        assert ratio <= 1.0, (mode, st, ratio)
    st1, st2 = results[az.ADAPTIVE_ANALYTIC_TILE][0], results[az.ADAPTIVE_ANALYTIC_PROBLEM][0]
    assert st1["sum_s"] + 33 * st1["native_tiles"] == st1["analytic_sum_s"]
    assert st2["sum_s"] + 33 * st2["native_tiles"] >= st1["sum_s"] + 33 * st1["native_tiles"]
    if phi >= 8.0:
        assert st1["native_tiles"] > 0


def test_probe_reruns_tiles_run_at_too_few_moduli(az):
    """an MLP that always answers s = 2 (on tiles whose analytic s stays below 23, so that no
    certificate takes them over): every tile is probed, fails and is rerun at its arbiter's s, and
    the result meets the target"""
    import torch
    m, n, k = 1030, 600, 700
    A, B = nn_problem(71, m, n, k, 1.0, 10)
    dA, dB = to_dev(A), to_dev(B)
    dC1 = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    az.set_mlp_weights(None)
    ref = az.gemm_adaptive([("N", "N", m, n, k, 1.5, dA, m, dB, k, 0.0, dC1, m, 16)], 53, az.ADAPTIVE_CERTIFIED_TILE)
    az.set_mlp_weights(const_class_params(0))
    try:
        dC0 = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.5, dA, m, dB, k, 0.0, dC0, m, 16)], 53, az.ADAPTIVE_MLP)
    finally:
        az.set_mlp_weights(None)
    assert st["mlp"] == 1
    assert st["probed"] == st["tiles"] and st["rerun"] == st["tiles"]
    assert st["rerun_sum_s"] == ref["analytic_sum_s"] == st["analytic_sum_s"]
    dC0 /= 1.5
    assert dd_check(az, m, n, k, dA, dB, dC0) <= 1.0


def smallest_s(az, dA, dB, m, n, k):
    import torch
    hi = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    az.dd_reference(m, n, k, dA, m, dB, k, hi, lo, ab)
    C = torch.empty(m * n, dtype=torch.float64, device="cuda")
    for s in range(2, 25):
        try:
            az.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, C, m, s)
        except ValueError:
            continue
        if az.error_ratio(m, n, k, C, m, hi, lo, ab) <= 1.0:
            return s
    return 25


def test_probe_passes_tiles_that_meet_the_target(az):
    """an MLP that answers the smallest sufficient s of the tile: the tile is probed (below its
    analytic s) and passes, with no rerun"""
    import torch
    m, n, k = TILE, TILE, 1024
    A, B = nn_problem(81, m, n, k, 0.0, 0)
    dA, dB = to_dev(A), to_dev(B)
    s_min = smallest_s(az, dA, dB, m, n, k)
    _, s_an = az.tile_features([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, torch.empty(1, device="cuda"), m, 16)])
    assert s_min < int(s_an[0]), "the analytic s is an upper bound with slack for uniform inputs"
    az.set_mlp_weights(const_class_params(s_min - 2))
    try:
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_MLP)
    finally:
        az.set_mlp_weights(None)
    # probed when s_min is below the arbiter (the certified s is within a modulus or two of s_min)
    assert st["analytic_sum_s"] >= s_min
    assert st["probed"] == (1 if st["analytic_sum_s"] > s_min else 0)
    assert st["rerun"] == 0 and st["sum_s"] == s_min
    assert dd_check(az, m, n, k, dA, dB, dC) <= 1.0


def test_mode0_without_weights_is_the_certified_tile_mode(az):
    import torch
    m, n, k = 800, 900, 333
    A, B = nn_problem(91, m, n, k, 3.0, 10)
    dA, dB = to_dev(A), to_dev(B)
    az.set_mlp_weights(None)
    out = []
    for mode in (az.ADAPTIVE_MLP, az.ADAPTIVE_CERTIFIED_TILE):
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, mode)
        out.append((st, dC))
    assert out[0][0]["mlp"] == 0 and out[0][0]["probed"] == 0
    assert out[0][0]["sum_s"] == out[1][0]["sum_s"]
    assert torch.equal(out[0][1].view(torch.int64), out[1][1].view(torch.int64))


def test_mlp_keeps_analytic_s_when_beta_is_nonzero(az):
    import torch
    m, n, k = 600, 600, 500
    A, B = nn_problem(95, m, n, k, 0.0, 0)
    dA, dB = to_dev(A), to_dev(B)
    az.set_mlp_weights(const_class_params(0))
    try:
        C0 = torch.ones(m * n, dtype=torch.float64, device="cuda")
        dC = C0.clone()
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.5, dC, m, 16)], 53, az.ADAPTIVE_MLP)
    finally:
        az.set_mlp_weights(None)
    assert st["probed"] == 0 and st["sum_s"] == st["analytic_sum_s"]
    dC1 = C0.clone()
    az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.5, dC1, m, 16)], 53, az.ADAPTIVE_CERTIFIED_TILE)
    assert torch.equal(dC.view(torch.int64), dC1.view(torch.int64))


def test_adaptive_early_returns_and_rejections(az):
    import torch
    C0 = torch.full((64 * 64,), 2.0, dtype=torch.float64, device="cuda")
    A = torch.ones(64 * 64, dtype=torch.float64, device="cuda")
    dC = C0.clone()
    az.gemm_adaptive([("N", "N", 64, 64, 64, 0.0, A, 64, A, 64, -0.5, dC, 64, 16),
                      ("N", "N", 0, 64, 64, 1.0, A, 64, A, 64, 0.0, dC, 64, 16)], 53, az.ADAPTIVE_ANALYTIC_TILE)
    torch.cuda.synchronize()
    assert torch.all(dC == -1.0)
    with pytest.raises(ValueError, match="problem 0"):
        az.gemm_adaptive([("N", "N", 64, 64, 64, 1.0, A, 0, A, 64, 0.0, dC, 64, 16)], 53, 1)
    with pytest.raises(ValueError):
        az.gemm_adaptive([("N", "N", 64, 64, 64, 1.0, A, 64, A, 64, 0.0, dC, 64, 16)], 53, 7)
    with pytest.raises(ValueError):
        az.set_adaptive_options(100, 0.9)


def test_default_model_loads_and_meets_the_target(az):
    """the shipped MLP: on fresh problems of the training distribution every output meets the
    target (probe and rerun included) with fewer moduli than the analytic rule"""
    import os
    import torch
    from oz2 import adaptive
    if not os.path.exists(adaptive.DEFAULT_MODEL):
        pytest.fail("the package ships no default MLP model")
    model = az.load_model()
    try:
        rng = np.random.default_rng(2024)
        total_s = total_an = 0
        for q in range(6):
            k = int(np.exp(rng.uniform(np.log(256), np.log(2048))))
            phi = float(rng.uniform(0, 8))
            m = n = k
            A, B = nn_problem(500 + q, m, n, k, phi, 40)
            dA, dB = to_dev(A), to_dev(B)
            dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
            st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_MLP)
            assert st["mlp"] == 1
            total_s += st["sum_s"] - st["rerun_sum_s"]
            total_an += st["analytic_sum_s"]
            assert dd_check(az, m, n, k, dA, dB, dC) <= 1.0, (q, k, phi, st)
        assert total_s <= total_an
        assert model["threshold"] > 0
    finally:
        az.set_mlp_weights(None)
        az.set_adaptive_options(TILE, 0.9)


def test_accuracy_metrics_match_the_oracle(oracle, az):
    """max ulp error and the correctly rounded count against the double-double product, on the
    device and by the oracle's restatement of the reference's accuracy bench"""
    import torch
    m, n, k = 300, 200, 700
    A, B = nn_problem(123, m, n, k, 2.0, 10)
    dA, dB = to_dev(A), to_dev(B)
    hi = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    az.dd_reference(m, n, k, dA, m, dB, k, hi, lo, ab)
    rn = hi + lo
    u, c = az.accuracy(m, n, rn, m, hi, lo)
    assert c == m * n and u <= 0.5
    for s in (10, 16):
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        az.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, s)
        u, c = az.accuracy(m, n, dC, m, hi, lo)
        want = oracle.metrics(dC.cpu().numpy(), hi.cpu().numpy(), lo.cpu().numpy())
        assert abs(u - want["ulp_max"]) <= 1e-6 * max(1.0, want["ulp_max"])
        assert c == round(want["cr_frac"] * m * n)


def test_native_tiles_keep_alpha_beta(az):
    """tiles sent to native FP64 (phi = 8, row offsets) with alpha and beta != 0: C is alpha A B +
    beta C within the DGEMM-level bound plus the rounding of the update"""
    import torch
    m, n, k = 900, 700, 800
    A, B = nn_problem(131, m, n, k, 8.0, 40)
    dA, dB = to_dev(A), to_dev(B)
    C0 = torch.rand(m * n, dtype=torch.float64, device="cuda") - 0.5
    dC = C0.clone()
    st = az.gemm_adaptive([("N", "N", m, n, k, -1.25, dA, m, dB, k, 0.75, dC, m, 16)], 53, az.ADAPTIVE_ANALYTIC_TILE)
    assert st["native_tiles"] > 0
    hi = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    az.dd_reference(m, n, k, dA, m, dB, k, hi, lo, ab)
    want = -1.25 * hi + 0.75 * C0
    err = (dC - want - (-1.25) * lo).abs()
    tol = 1.25 * k * 2.0 ** -53 * ab + 2.0 ** -51 * (want.abs() + (0.75 * C0).abs()) + 1e-300
    assert bool((err <= tol).all())


def test_ops_do_not_change_adaptive_results(az):
    """mode 1 with op(A) = T and op(B) = T on explicitly transposed copies equals the NN call bit
    for bit (statistics, features and s are functions of op(A) rows and op(B) columns)"""
    import torch
    m, n, k = 700, 1100, 600
    A, B = nn_problem(141, m, n, k, 3.0, 20)
    dA, dB = to_dev(A), to_dev(B)
    dAt, dBt = to_dev(np.asfortranarray(A.T)), to_dev(np.asfortranarray(B.T))
    out = []
    for ta, tb, AA, lda, BB, ldb in (("N", "N", dA, m, dB, k), ("T", "T", dAt, k, dBt, n), ("T", "N", dAt, k, dB, k)):
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([(ta, tb, m, n, k, 1.0, AA, lda, BB, ldb, 0.0, dC, m, 16)], 53, az.ADAPTIVE_ANALYTIC_TILE)
        out.append((st["sum_s"], st["native_tiles"], dC))
    for s_, nat, c in out[1:]:
        assert s_ == out[0][0] and nat == out[0][1]
        assert torch.equal(c.view(torch.int64), out[0][2].view(torch.int64))


def test_whole_problem_and_tile_tasks_agree(az):
    """a problem whose tiles share one s runs as one task unless the workspace limit forbids it;
    both ways give the same bits"""
    import torch
    import oz2
    m = n = 2048
    k = 1024
    A, B = nn_problem(151, m, n, k, 1.0, 10)
    dA, dB = to_dev(A), to_dev(B)
    out = []
    for limit in (0, 200 << 20):
        h = oz2.Ozaki2(torch.cuda.current_stream())
        try:
            h.set_workspace_limit(limit)
            dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
            h.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_FIXED)
            torch.cuda.synchronize()
            out.append(dC)
        finally:
            h.close()
    assert torch.equal(out[0].view(torch.int64), out[1].view(torch.int64))
    dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    az.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)
    assert torch.equal(out[0].view(torch.int64), dC.view(torch.int64))


@pytest.mark.parametrize("m,n,k,phi,offsets", [(700, 900, 600, 0.0, 0), (1030, 600, 777, 3.0, 20),
                                               (600, 1100, 1500, 6.0, 40), (520, 520, 300, 8.0, 40)])
def test_certified_modes_meet_the_target(az, m, n, k, phi, offsets):
    """modes 4 (certified s per tile) and 5 (per problem): every output within the target, the
    arbiter never above the analytic rule, the same result on every run, and op(A) = T / op(B) = T
    on explicitly transposed copies (the k-contiguous certificate layouts) equal to NN bit for bit"""
    import torch
    A, B = nn_problem(300 + m, m, n, k, phi, offsets)
    dA, dB = to_dev(A), to_dev(B)
    dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    an = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_ANALYTIC_TILE)
    outs = []
    for mode in (az.ADAPTIVE_CERTIFIED_TILE, az.ADAPTIVE_CERTIFIED_PROBLEM, az.ADAPTIVE_CERTIFIED_TILE):
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, mode)
        assert dd_check(az, m, n, k, dA, dB, dC) <= 1.0, (mode, st)
        assert st["analytic_sum_s"] <= an["analytic_sum_s"]
        assert st["probed"] == 0 and st["mlp"] == 0
        outs.append((st, dC))
    assert torch.equal(outs[0][1].view(torch.int64), outs[2][1].view(torch.int64))
    At = to_dev(np.asfortranarray(A.T))  # k x m: op(A) = T gives A
    Bt = to_dev(np.asfortranarray(B.T))  # n x k
    dT = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    az.gemm_adaptive([("T", "T", m, n, k, 1.0, At, k, Bt, n, 0.0, dT, m, 16)], 53, az.ADAPTIVE_CERTIFIED_TILE)
    assert torch.equal(dT.view(torch.int64), outs[0][1].view(torch.int64))
    if phi >= 6.0:
        assert outs[0][0]["native_tiles"] <= an["native_tiles"]


@pytest.mark.parametrize("seed,n,k,phi", [(1, 300, 400, 0.0), (2, 512, 1000, 2.5), (3, 256, 2000, 4.0),
                                          (4, 400, 333, 6.0), (5, 512, 512, 1.0), (6, 500, 700, 5.0),
                                          (7, 384, 1500, 7.0)])
def test_certified_s_matches_the_restatement(oracle, az, seed, n, k, phi):
    """one tile per problem: where the analytic s is 23 or more the device's arbiter lies between
    the restated certificate (FP64 |A||B|) and one modulus above it (the device's bf16 lower
    bound is a little smaller); below 23 no certificate runs and the arbiter is the analytic s"""
    import torch
    A, B = nn_problem(700 + seed, n, n, k, phi, 30)
    dA, dB = to_dev(A), to_dev(B)
    dC = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    st = az.gemm_adaptive([("N", "N", n, n, k, 1.0, dA, n, dB, k, 0.0, dC, n, 16)], 53, az.ADAPTIVE_CERTIFIED_TILE)
    assert st["tiles"] == 1
    s_np = adaptive_oracle.certified_s(oracle, A, B)
    _, s_an = adaptive_oracle.tile_features(oracle, [("N", "N", n, n, k, A, B)])
    if int(s_an[0]) < 23:
        assert st["analytic_sum_s"] == int(s_an[0])
        return
    lo_s, hi_s = min(int(s_an[0]), s_np), min(int(s_an[0]), s_np + 1)
    assert lo_s <= st["analytic_sum_s"] <= hi_s, (st, s_np, int(s_an[0]))


def test_certified_tiles_override_the_mlp(az):
    """an MLP that always answers s = 2 on heavy-tailed inputs (analytic s 23 or more): the
    certified tiles take their certificate and are not probed, and every output meets the target"""
    import torch
    m, n, k = 1030, 600, 700
    A, B = nn_problem(171, m, n, k, 5.0, 40)
    dA, dB = to_dev(A), to_dev(B)
    ref = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, torch.zeros(m * n, dtype=torch.float64,
                                                                                    device="cuda"), m, 16)],
                           53, az.ADAPTIVE_CERTIFIED_TILE)
    az.set_mlp_weights(const_class_params(0))
    try:
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_MLP)
    finally:
        az.set_mlp_weights(None)
    assert st["mlp"] == 1 and st["probed"] == 0
    assert st["sum_s"] == ref["sum_s"] and st["native_tiles"] == ref["native_tiles"]
    assert dd_check(az, m, n, k, dA, dB, dC) <= 1.0


def test_results_do_not_depend_on_concurrent_host_copies(az):
    """the call's own transfers (item tables in through the pinned ring, tile decisions out) run as
    copy kernels on an internal stream: with large host copies queued on two other streams the
    outputs are the same bits as without them, in the MLP mode (probe reads included) and the
    certified tile mode, on a batch whose item tables exceed one kernel-parameter blob"""
    import torch
    model = az.load_model()
    try:
        rng = np.random.default_rng(77)
        probs, outs = [], []
        for q in range(16):
            n = int(rng.integers(300, 1400))
            A, B = nn_problem(900 + 2 * q, n, n, n, float(rng.uniform(0, 8)), 40)
            probs.append((n, to_dev(A), to_dev(B)))

        def run(mode):
            Cs = [torch.zeros(n * n, dtype=torch.float64, device="cuda") for n, _, _ in probs]
            az.gemm_adaptive([("N", "N", n, n, n, 1.0, dA, n, dB, n, 0.0, dC, n, 16)
                              for (n, dA, dB), dC in zip(probs, Cs)], 53, mode)
            return Cs

        big = 1 << 26  # 512 MiB each way
        h_in = torch.ones(big, dtype=torch.float64, pin_memory=True)
        h_out = torch.empty(big, dtype=torch.float64, pin_memory=True)
        d_in = torch.empty(big, dtype=torch.float64, device="cuda")
        d_out = torch.ones(big, dtype=torch.float64, device="cuda")
        up, down = torch.cuda.Stream(), torch.cuda.Stream()
        for mode in (az.ADAPTIVE_MLP, az.ADAPTIVE_CERTIFIED_TILE):
            quiet = run(mode)
            torch.cuda.synchronize()
            for _ in range(3):
                with torch.cuda.stream(up):
                    d_in.copy_(h_in, non_blocking=True)
                with torch.cuda.stream(down):
                    h_out.copy_(d_out, non_blocking=True)
            busy = run(mode)
            torch.cuda.synchronize()
            az.check_device_error()
            for (n, _, _), a, b in zip(probs, quiet, busy):
                assert torch.equal(a.view(torch.int64), b.view(torch.int64)), (mode, n)
        assert model["threshold"] > 0
    finally:
        az.set_mlp_weights(None)
        az.set_adaptive_options(TILE, 0.9)


def test_gemm_bytes_count_planes_once_and_residues(az):
    """the algorithmic bytes of the adaptive call's INT8 GEMM: each split panel's planes read once
    (rows padded to 256 / 128, k to 128) and s m n residue bytes written (rows padded to 32)"""
    m = n = 512
    k, s = 700, 16
    A = make_mat(61, m, k, m, "u")
    B = make_mat(62, k, n, k, "u")
    C0 = make_mat(63, m, n, m, "u")
    az.gemm_adaptive([("N", "N", m, n, k, 1.0, to_dev(A), m, to_dev(B), k, 0.0, to_dev(C0), m, s)], 53,
                     az.ADAPTIVE_FIXED)
    kp = math.ceil(k / 128) * 128
    got = az.adaptive_gemm_bytes()
    assert got == {"plane_bytes": s * (512 * kp + 512 * kp), "residue_bytes": s * m * n, "batches": 1}


@pytest.mark.parametrize("kind", [1, 2])
def test_freivalds_probe_reruns_tiles_run_at_too_few_moduli(az, kind):
    """the Freivalds test (C x against alpha A (B x) in double-double), alone and beside the column
    probe: an MLP that always answers s = 2 leaves every tile far off, every tile fails and is rerun
    at its arbiter's s, and the result meets the target"""
    import torch
    m, n, k = 1030, 600, 700
    A, B = nn_problem(73, m, n, k, 1.0, 10)
    dA, dB = to_dev(A), to_dev(B)
    az.set_mlp_weights(const_class_params(0))
    az.set_probe_kind(kind)
    try:
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.5, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_MLP)
    finally:
        az.set_mlp_weights(None)
        az.set_probe_kind(0)
    assert st["probed"] == st["tiles"] and st["rerun"] == st["tiles"]
    dC /= 1.5
    assert dd_check(az, m, n, k, dA, dB, dC) <= 1.0


@pytest.mark.parametrize("phi,offsets", [(0.0, 0), (1.0, 10)])
def test_freivalds_probe_passes_tiles_that_meet_the_target(az, phi, offsets):
    """a tile run at its smallest sufficient s meets the target entry by entry, so the Freivalds
    test (whose per-row tolerance is the target summed with the weights |x_j|) must pass it"""
    import torch
    m, n, k = TILE, TILE, 1024
    A, B = nn_problem(83, m, n, k, phi, offsets)
    dA, dB = to_dev(A), to_dev(B)
    s_min = smallest_s(az, dA, dB, m, n, k)
    dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    arbiter = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53,
                             az.ADAPTIVE_CERTIFIED_TILE)["analytic_sum_s"]
    _, s_an = az.tile_features([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)])
    assert int(s_an[0]) < 23, "a tile the certificate would take over is never probed"
    if s_min >= arbiter or s_min > 24:
        pytest.skip("no s below the arbiter's meets the target here: nothing to probe")
    az.set_mlp_weights(const_class_params(s_min - 2))
    az.set_probe_kind(1)
    try:
        dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
        st = az.gemm_adaptive([("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, dC, m, 16)], 53, az.ADAPTIVE_MLP)
    finally:
        az.set_mlp_weights(None)
        az.set_probe_kind(0)
    assert st["probed"] == 1 and st["rerun"] == 0 and st["sum_s"] == s_min
    assert dd_check(az, m, n, k, dA, dB, dC) <= 1.0


def test_probe_kind_is_checked(az):
    with pytest.raises(ValueError):
        az.set_probe_kind(4)


@pytest.mark.parametrize("s", range(25, 33))
def test_extended_moduli_match_the_oracle(oracle, az, s):
    """the adaptive path's own moduli sets (s = 25..32, up to 124 bits per element: the four-word
    split and CRTs of 7 and 8 limbs) equal the oracle's restatement bit for bit (mode 3 runs each
    problem at its own s), for all op pairs, alpha / beta, padded leading dimensions and wide
    exponent ranges; every result is inside the rigorous bound"""
    import torch
    cases = [("N", "N", 300, 200, 777), ("T", "N", 130, 257, 1500), ("N", "T", 64, 90, 40), ("T", "T", 200, 150, 3000)]
    ta, tb, m, n, k = cases[s % len(cases)]
    Ar, Ac = op_shape(ta, m, k)
    Br, Bc = op_shape(tb, k, n)
    A = make_mat(100 + s, Ar, Ac, Ar + 2, "wide", 30)
    B = make_mat(200 + s, Br, Bc, Br + 1, "wide", 30)
    C0 = make_mat(300 + s, m, n, m + 3, "u")
    dC = to_dev(C0)
    az.gemm_adaptive([(ta, tb, m, n, k, 1.5, to_dev(A), Ar + 2, to_dev(B), Br + 1, -0.5, dC, m + 3, s)], 53,
                     az.ADAPTIVE_FIXED)
    torch.cuda.synchronize()
    az.check_device_error()
    want = C0.copy(order="F")
    assert oracle.dgemm_ext(ta, tb, m, n, k, 1.5, A, Ar + 2, B, Br + 1, -0.5, want, m + 3, s) == 0
    got = from_dev(dC, C0)
    nd = int((bits(got) != bits(want)).sum())
    assert nd == 0, f"{nd} entries differ from the oracle at s = {s}"
    tk = oracle.plan_ext(s, k).tk
    assert tk > 85  # beyond every plan of s <= 24 at this k
    if s in (26, 32):
        assert tk > 92  # the split's four-word path

