"""numpy restatement of the adaptive-s tile statistics: the exponent-gap histogram of each panel,
the sixteen tile features and the analytic number of moduli per C tile.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's reference leg (to pick the
per-problem analytic s the reference's CPU path runs at), never by the product package.

Definitions (no counterpart in the reference, whose number of moduli is fixed per call):
  gap of a nonzero finite x in a row = frexp exponent of the row maximum - frexp exponent of x,
  clamped to [0, 63]; rows whose maximum is zero or non-finite contribute nothing; zeros are
  counted apart.
  analytic s = the smallest s in 2..24 whose bits per element tk (the plan of the reference's
  Ozaki2::gemm for this k) reach R + 2 + t - floor(log2(k - 1)), R the largest gap of the tile's
  two panels, t the target bits, over s = 2..32 (the library's extended sets above 24); 33 (the
  tile runs as a native FP64 GEMM) when none does or when R reaches the last gap bin (63: every
  gap of 63 binades or more, which bounds nothing).
"""
import math

import numpy as np

TILE = 512
MAX_S = 32   # the library's extended moduli sets reach s = 32 in the adaptive path
NATIVE = 33  # the s of a tile run as a native FP64 GEMM
QUANTILES = (0.5, 0.75, 0.9, 0.99)


def _frexp_e(x):
    return np.frexp(x)[1].astype(np.int64)


def panel_stats(X):
    """X: (rows, k) with the rows of op(A) (or the columns of op(B)) as rows.
    Returns (hist[65], exponent spread of the row maxima)."""
    ax = np.abs(X)
    mx = ax.max(axis=1) if ax.shape[1] else np.zeros(ax.shape[0])
    live = (mx > 0) & np.isfinite(mx)
    hist = np.zeros(65, dtype=np.int64)
    Y = ax[live]
    em = _frexp_e(mx[live])
    nz = (Y != 0) & np.isfinite(Y)
    gaps = np.clip(em[:, None] - _frexp_e(np.where(nz, Y, 1.0)), 0, 63)[nz]
    hist[:64] = np.bincount(gaps, minlength=64)
    hist[64] = (Y == 0).sum()
    spread = float(em.max() - em.min()) if em.size else 0.0
    return hist, spread


def gap_quantile(h, q):
    nz = int(h[:64].sum())
    if nz == 0:
        return 0.0
    want = int(np.float64(np.float32(q)) * float(nz - 1)) + 1
    return float(np.argmax(np.cumsum(h[:64]) >= want))


def floor_log2_km1(k):
    lg, v = 0, k - 1
    while v > 1:
        v >>= 1
        lg += 1
    return lg


def tk_table(oracle, k):
    tk = [0] * (MAX_S + 1)
    for s in range(2, MAX_S + 1):
        try:
            tk[s] = oracle.plan_ext(s, k).tk
        except ValueError:
            tk[s] = 0
    return tk


def analytic_s(tk, R, k, target_bits=53):
    need = R + 2 + target_bits - floor_log2_km1(k)
    if R >= 63:
        return NATIVE
    return next((s for s in range(2, MAX_S + 1) if tk[s] >= need), NATIVE)


def tile_features(oracle, problems, target_bits=53, tile=TILE):
    """problems: (ta, tb, m, n, k, A, B) with column-major numpy A, B (stored shapes). Returns the
    features (float32 [tiles, 18]) and analytic s ([tiles]), column tiles outer, row tiles inner."""
    out_f, out_s = [], []
    for (ta, tb, m, n, k, A, B) in problems:
        opA = A[:m, :k] if ta == "N" else A[:k, :m].T
        opB = B[:k, :n] if tb == "N" else B[:n, :k].T
        tk = tk_table(oracle, k)
        for J in range(0, n, tile):
            hb, sb = panel_stats(opB[:, J:J + tile].T)
            for I in range(0, m, tile):
                ha, sa = panel_stats(opA[I:I + tile, :])
                f = np.zeros(18, dtype=np.float32)
                f[0] = np.float32(np.log2(np.float32(k))) / 16
                f[1] = np.float32(target_bits) / 64
                for q, qq in enumerate(QUANTILES):
                    f[2 + q] = gap_quantile(ha, qq) / 64
                    f[8 + q] = gap_quantile(hb, qq) / 64
                ra = int(np.nonzero(ha[:64])[0].max()) if ha[:64].any() else 0
                rb = int(np.nonzero(hb[:64])[0].max()) if hb[:64].any() else 0
                f[6], f[12] = ra / 64, rb / 64
                f[7] = np.float32(ha[64] / float(ha.sum())) if ha.sum() else 0
                f[13] = np.float32(hb[64] / float(hb.sum())) if hb.sum() else 0
                f[14], f[15] = sa / 64, sb / 64
                f[16] = np.float32(min(tile, m - I)) / np.float32(512)
                f[17] = np.float32(min(tile, n - J)) / np.float32(512)
                out_f.append(f)
                out_s.append(analytic_s(tk, max(ra, rb), k, target_bits))
    return np.array(out_f).reshape(-1, 18), np.array(out_s, dtype=np.int64)


def problem_analytic_s(oracle, ta, tb, m, n, k, A, B, target_bits=53, tile=TILE):
    """the largest analytic s over the problem's tiles (the per-problem fixed analytic s)"""
    return int(tile_features(oracle, [(ta, tb, m, n, k, A, B)], target_bits, tile)[1].max())


def certified_s(oracle, opA, opB, target_bits=53):
    """certified s of one tile: op(A) (m x k) and op(B) (k x n) as numpy arrays, restating the
    entrywise a-priori bound of the library's certificate with the FP64 product |op(A)||op(B)| in
    place of its bf16 lower bound (so the library's s is this one or above). 33 when no s <= 32
    reaches it, the two roundings use up the target or an input is non-finite."""
    k = opA.shape[1]
    t = float(target_bits)
    Bu = k - 2.0 ** (t - 52.0)
    if Bu <= 0 or not (np.all(np.isfinite(opA)) and np.all(np.isfinite(opB))):
        return NATIVE
    ma, mb = np.abs(opA).max(axis=1), np.abs(opB).max(axis=0)
    e = np.where(ma > 0, np.frexp(ma)[1], 0)
    f = np.where(mb > 0, np.frexp(mb)[1], 0)
    Ra = np.abs(opA).sum(axis=1) * np.ldexp(1.0, -e)
    Sb = np.abs(opB).sum(axis=0) * np.ldexp(1.0, -f)
    G = (np.abs(opA) @ np.abs(opB)) * np.ldexp(1.0, -e)[:, None] * np.ldexp(1.0, -f)[None, :]
    live = (Ra[:, None] > 0) & (Sb[None, :] > 0)
    if not np.any(live):
        return 2
    if np.any(G[live] == 0):
        return NATIVE
    q1 = ((Ra[:, None] + Sb[None, :]) / np.where(live, G, 1.0))[live].max()
    q2 = (1.0 / np.where(live, G, 1.0))[live].max()
    c = 1.0 - 2.0 ** -6
    l1 = math.log2(q1 * (1 + 2.0 ** -20)) + t - 1.0 - math.log2(Bu * c * (1 - 2.0 ** -10))
    l2 = 0.5 * (math.log2(q2 * (1 + 2.0 ** -20)) + t + 10.0 - math.log2(Bu / k * c))
    need = math.ceil(max(l1, l2) + 1e-9)
    tk = tk_table(oracle, k)
    return next((s for s in range(2, MAX_S + 1) if tk[s] > 0 and tk[s] >= need), NATIVE)
