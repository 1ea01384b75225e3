"""The grouped launch (many DGEMMs of uneven m, n, k, ops and s in one set of launches): its
results equal those of separate Ozaki2::gemm calls bit for bit, under every GEMM configuration,
with CUDA-graph replay, and with k chunks inside the group."""
import numpy as np
import pytest

from common import bits, from_dev, make_mat, op_shape, to_dev

pytestmark = pytest.mark.gpu


def make_group(seed, count, lo=32, hi=700, s_range=(14, 20), kmax=None):
    rng = np.random.default_rng(seed)
    probs = []
    for q in range(count):
        m, n, k = (int(np.exp(rng.uniform(np.log(lo), np.log(hi)))) for _ in range(3))
        if kmax:
            k = min(k, kmax)
        ta, tb = rng.choice(list("NT")), rng.choice(list("NT"))
        s = int(rng.integers(s_range[0], s_range[1] + 1))
        Ar, Ac = op_shape(ta, m, k)
        Br, Bc = op_shape(tb, k, n)
        A = make_mat(seed * 1000 + 3 * q, Ar, Ac, Ar + q % 3, "wide", 6)
        B = make_mat(seed * 1000 + 3 * q + 1, Br, Bc, Br + q % 2, "wide", 6)
        C0 = make_mat(seed * 1000 + 3 * q + 2, m, n, m + q % 4, "u")
        probs.append(dict(ta=ta, tb=tb, m=m, n=n, k=k, s=s, alpha=[1.0, -0.75, 2.0][q % 3],
                          beta=[0.0, 0.5, -1.0][q % 3], A=A, B=B, C0=C0))
    return probs


def device(probs):
    return [dict(p, dA=to_dev(p["A"]), dB=to_dev(p["B"]), dC=to_dev(p["C0"])) for p in probs]


def args(p, C_=None):
    return (p["ta"], p["tb"], p["m"], p["n"], p["k"], p["alpha"], p["dA"], p["A"].shape[0], p["dB"],
            p["B"].shape[0], p["beta"], C_ if C_ is not None else p["dC"], p["C0"].shape[0], p["s"])


def singles(oz, probs):
    import torch
    out = []
    for p in probs:
        dC = to_dev(p["C0"])
        oz.gemm(*args(p, dC))
        torch.cuda.synchronize()
        out.append(from_dev(dC, p["C0"]))
    return out


def grouped(oz, probs):
    import torch
    for p in probs:
        p["dC"].copy_(to_dev(p["C0"]))
    oz.gemm_grouped([args(p) for p in probs])
    torch.cuda.synchronize()
    oz.check_device_error()
    return [from_dev(p["dC"], p["C0"]) for p in probs]


def test_grouped_equals_single_calls(oz):
    probs = device(make_group(1, 40))
    want = singles(oz, probs)
    got = grouped(oz, probs)
    for q, (g, w) in enumerate(zip(got, want)):
        assert np.array_equal(bits(g), bits(w)), f"problem {q}"


def test_grouped_matches_oracle(oracle, oz):
    probs = device(make_group(2, 6, hi=300))
    got = grouped(oz, probs)
    for p, g in zip(probs, got):
        Co = p["C0"].copy(order="F")
        assert oracle.dgemm(p["ta"], p["tb"], p["m"], p["n"], p["k"], p["alpha"], p["A"], p["A"].shape[0], p["B"],
                            p["B"].shape[0], p["beta"], Co, Co.shape[0], p["s"]) == 0
        assert np.array_equal(bits(g), bits(Co))


@pytest.mark.parametrize("bn,group_j,ctas", [(128, 4, 0), (256, 32, 0), (128, 16, 37)])
def test_grouped_every_config_bit_identical(oz, bn, group_j, ctas):
    probs = device(make_group(3, 24))
    want = singles(oz, probs)
    oz.set_gemm_config(bn, group_j, ctas)
    try:
        got = grouped(oz, probs)
        assert oz.gemm_config() == {"bn": bn, "group_j": group_j, "ctas": ctas}
    finally:
        oz.set_gemm_config(0)
    for g, w in zip(got, want):
        assert np.array_equal(bits(g), bits(w))


def test_grouped_graph_replay_follows_new_data(oz):
    import torch
    probs = device(make_group(4, 16))
    oz.set_graph_mode(True)
    try:
        first = grouped(oz, probs)  # captured
        again = grouped(oz, probs)  # replayed
        for a, b in zip(first, again):
            assert np.array_equal(bits(a), bits(b))
        # same buffers, new values: the replayed graph must compute the new products
        for q, p in enumerate(probs):
            p["A"] = np.asfortranarray(p["A"] * 0.5 + 0.125)
            p["dA"].copy_(to_dev(p["A"]))
        replayed = grouped(oz, probs)
    finally:
        oz.set_graph_mode(False)
    want = singles(oz, probs)
    for g, w in zip(replayed, want):
        assert np.array_equal(bits(g), bits(w))


def test_autotune_picks_a_valid_config_and_keeps_results(oz):
    probs = device(make_group(5, 20))
    want = singles(oz, probs)
    cfg = oz.autotune_grouped([args(p) for p in probs])
    assert cfg["bn"] in (128, 256) and cfg["group_j"] >= 1
    got = grouped(oz, probs)
    assert oz.gemm_config()["bn"] == cfg["bn"]
    for g, w in zip(got, want):
        assert np.array_equal(bits(g), bits(w))


def test_grouped_with_k_chunks_and_early_returns(oracle, oz):
    import torch
    probs = make_group(6, 3, hi=64)
    probs[1]["k"] = 140000
    ta, tb = probs[1]["ta"], probs[1]["tb"]
    Ar, Ac = op_shape(ta, probs[1]["m"], 140000)
    Br, Bc = op_shape(tb, 140000, probs[1]["n"])
    probs[1]["A"] = make_mat(61, Ar, Ac, Ar, "wide", 2)
    probs[1]["B"] = make_mat(62, Br, Bc, Br, "wide", 2)
    probs[2]["alpha"] = 0.0  # C = beta C
    probs = device(probs)
    got = grouped(oz, probs)
    for p, g in zip(probs, got):
        Co = p["C0"].copy(order="F")
        oracle.dgemm(p["ta"], p["tb"], p["m"], p["n"], p["k"], p["alpha"], p["A"], p["A"].shape[0], p["B"],
                     p["B"].shape[0], p["beta"], Co, Co.shape[0], p["s"])
        assert np.array_equal(bits(g), bits(Co))


def test_grouped_rejects_bad_problem_before_running(oz):
    import torch
    probs = device(make_group(7, 3, hi=64))
    bad = list(args(probs[1]))
    bad[7] = 0  # lda
    before = [p["dC"].clone() for p in probs]
    with pytest.raises(ValueError, match="problem 1"):
        oz.gemm_grouped([args(probs[0]), tuple(bad), args(probs[2])])
    torch.cuda.synchronize()
    for p, b in zip(probs, before):
        assert torch.equal(p["dC"], b)
