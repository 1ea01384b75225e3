"""CPU checks of the adaptive-s pieces that need no device: the numpy restatement of the tile
statistics on hand-computed cases, and the shipped MLP model file."""
import json
import os

import numpy as np

import adaptive_oracle as ao
from common import ROOT


def test_gap_histogram_by_hand():
    # row 0: max 4 (frexp exponent 3); 1 -> gap 2, 0.5 -> gap 3, 0 counted apart, 2^-70 -> 63 (clamped)
    # row 1: all zero, contributes nothing
    X = np.array([[4.0, 1.0, -0.5, 0.0, 2.0 ** -70], [0.0] * 5])
    h, spread = ao.panel_stats(X)
    want = np.zeros(65, dtype=np.int64)
    want[0], want[2], want[3], want[63], want[64] = 1, 1, 1, 1, 1
    assert np.array_equal(h, want)
    assert spread == 0.0
    # want = floor(q (nonzero - 1)) + 1 of the 4 nonzero gaps (0, 2, 3, 63)
    assert ao.gap_quantile(h, 0.5) == 2.0 and ao.gap_quantile(h, 0.99) == 3.0 and ao.gap_quantile(h, 1.0) == 63.0


def test_subnormal_gaps_use_the_true_exponent():
    X = np.array([[1.0, 2.0 ** -1074, 2.0 ** -1030]])
    h, _ = ao.panel_stats(X)
    assert h[63] == 2 and h[0] == 1


def test_analytic_s_rule(oracle):
    k = 1024
    tk = ao.tk_table(oracle, k)
    # R = 0: need tk >= 2 + 53 - 9 = 46
    s0 = ao.analytic_s(tk, 0, k)
    assert tk[s0] >= 46 and tk[s0 - 1] < 46
    # the last gap bin (63 binades or more) bounds nothing: native FP64
    assert ao.analytic_s(tk, 63, k) == ao.NATIVE == 33
    # beyond what 24 moduli give: the extended sets (tk 85 at s = 24 for k = 1024)
    s1 = ao.analytic_s(tk, 45, k)
    assert 24 < s1 <= 32 and tk[s1] >= 45 + 2 + 53 - 9 > tk[24]
    # the extended plans follow the reference's tk rule, with M from the library's own sets
    for s in range(25, 33):
        p = oracle.plan_ext(s, k)
        assert p.tk == tk[s] and k * 2 ** (2 * p.tk + 2) <= p.Mint < k * 2 ** (2 * p.tk + 4)
    assert ao.floor_log2_km1(1) == 0 and ao.floor_log2_km1(2) == 0 and ao.floor_log2_km1(1025) == 10


def test_tile_order_and_edges(oracle):
    rng = np.random.default_rng(1)
    A = np.asfortranarray(rng.standard_normal((700, 40)))
    B = np.asfortranarray(rng.standard_normal((40, 600)))
    f, s = ao.tile_features(oracle, [("N", "N", 700, 600, 40, A, B)])
    assert f.shape == (4, 18) and s.shape == (4,)
    # rows / columns of each tile over 512: tiles (0,0) (1,0) (0,1) (1,1)
    assert np.allclose(f[:, 16], [1.0, 188 / 512, 1.0, 188 / 512]) and np.allclose(f[:, 17], [1, 1, 88 / 512, 88 / 512])
    assert np.all(f[:, 0] == np.float32(np.log2(np.float32(40))) / 16)


def test_shipped_model_file():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "os2-xe_b200"))
    path = os.path.join(ROOT, "os2-xe_b200", "oz2", "adaptive_mlp.json")
    with open(path) as fh:
        model = json.load(fh)
    # parameter count of the 18 -> 32 -> 32 -> 24 MLP (classes s = 2..24 and native FP64)
    assert len(model["params"]) == 32 * 18 + 32 + 32 * 32 + 32 + 24 * 32 + 24
    assert all(np.isfinite(model["params"]))
    assert 0 < model["threshold"] <= 1 and model["tile"] % 128 == 0
