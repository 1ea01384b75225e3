"""Accuracy of the emulated DGEMM / ZGEMM against a double-double product, one CSV row per
(distribution, k, method, s): the rows and columns of the reference's accuracy bench
(benchmarks/bench_accuracy.cpp:190-285), with this library's emulation (`ozaki2`,
`ozaki2_3m`) beside native cuBLAS (`dgemm_gpu`, `zgemm_gpu`) and the Ozaki Scheme I baseline
(`ozaki1`, real only: the s column holds its L (L + 1) / 2 GEMMs, tk = 7 L - 2, as the reference's
rows do, :256-261).

    python -m oz2.bench_accuracy [--k 256,1024,4096] [--s 4-24] [--L 4-9]
                                 [--dist urand,phi0.5,phi2,phi4] [--mn 512] [--complex] [--seed 1]

Distributions (m = n = mn, inner dimension k; the same definitions as the reference's `gen`,
seeded here by numpy's PCG64, so the values differ):
  urand   U[-1, 1)
  phiX    (u - 0.5) exp(X g), u ~ U[0, 1), g ~ N(0, 1)
  sincos  A_rc = sin(r + c), B_rc = cos(r c)
  spike   urand, and one entry per row of A (column 7919 r mod k) scaled by 2^40
  cancel  urand; the second half of A's columns repeats the first, the second half of B's rows is
          minus the first plus 2^-30 of itself: most of each product cancels
Metrics per row (the reference's `measure`, :69-94): ulp_max and ulp_mean of |C - (hi + lo)| in
units of the spacing above |hi|, cr_frac the fraction of entries equal to RN(hi + lo), ab_max =
max |C - (hi + lo)| / (|A||B|), fro_rel = ||C - (hi + lo)||_F / ||hi||_F.
"""
import argparse
import math
import sys

import numpy as np

CSV_HEADER = "dist,k,method,s,tk,ulp_max,ulp_mean,cr_frac,ab_max,fro_rel"


def parse_ints(text):
    out = []
    for part in text.split(","):
        if "-" in part:
            a, b = part.split("-")
            out.extend(range(int(a), int(b) + 1))
        elif part:
            out.append(int(part))
    return out


def generate(rows, cols, dist, seed, is_a):
    """column-major (rows x cols) float64 numpy array of the named distribution"""
    rng = np.random.default_rng(seed)
    if dist in ("urand", "spike", "cancel"):
        X = 2.0 * rng.random((rows, cols)) - 1.0
    elif dist == "sincos":
        r = np.arange(rows, dtype=np.float64)[:, None]
        c = np.arange(cols, dtype=np.float64)[None, :]
        X = np.sin(r + c) if is_a else np.cos(r * c)
    elif dist.startswith("phi"):
        phi = float(dist[3:])
        X = (rng.random((rows, cols)) - 0.5) * np.exp(phi * rng.standard_normal((rows, cols)))
    else:
        raise ValueError(f"unknown distribution {dist}")
    if dist == "spike" and is_a:
        r = np.arange(rows)
        X[r, (r * 7919) % cols] *= 2.0 ** 40
    if dist == "cancel":
        if is_a:
            h = cols // 2
            X[:, h:2 * h] = X[:, :h]
        else:
            h = rows // 2
            X[h:2 * h, :] = -X[:h, :] + np.ldexp(X[h:2 * h, :], -30)
    return np.asfortranarray(X)


def metrics(torch, C, hi, lo, absab):
    """the reference's five accuracy figures from device tensors (flat, equal lengths)"""
    err = ((C - hi) - lo).abs()
    ahi = hi.abs()
    ulp = torch.nextafter(ahi, torch.full_like(ahi, math.inf)) - ahi
    ulp = torch.where(hi == 0, torch.full_like(ulp, 4.9406564584124654e-324), ulp)
    eu = err / ulp
    pos = absab > 0
    ab = (err[pos] / absab[pos]).max().item() if bool(pos.any()) else 0.0
    r2 = (hi * hi).sum().item()
    return (eu.max().item(), eu.mean().item(), (C == hi + lo).double().mean().item(), ab,
            math.sqrt((err * err).sum().item() / r2) if r2 > 0 else 0.0)


def row(dist, k, method, s, tk, m5):
    return "%s,%d,%s,%d,%d,%.4g,%.4g,%.6f,%.4g,%.4g" % ((dist, k, method, s, tk) + tuple(m5))


def run_real(oz, torch, dist, k, mn, svals, seed, Ls=()):
    import oz2
    m = n = mn
    A = generate(m, k, dist, seed * 1000 + 11 + k, True)
    B = generate(k, n, dist, seed * 1000 + 77 + k, False)
    dA = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    dB = torch.from_numpy(B.ravel(order="F").copy()).cuda()
    hi = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    oz.dd_reference(m, n, k, dA, m, dB, k, hi, lo, ab)
    out = []
    C = torch.mm(dB.view(n, k), dA.view(k, m)).reshape(-1)  # C^T row-major = C column-major
    out.append(row(dist, k, "dgemm_gpu", 0, 53, metrics(torch, C, hi, lo, ab)))
    C = torch.empty(m * n, dtype=torch.float64, device="cuda")
    for s in svals:
        try:
            tk = oz2.Ozaki2.precision_bits(k, s)
        except ValueError:
            continue
        oz.gemm("N", "N", m, n, k, 1.0, dA, m, dB, k, 0.0, C, m, s)
        out.append(row(dist, k, "ozaki2", s, tk, metrics(torch, C, hi, lo, ab)))
    for L in Ls:
        try:
            oz.ozaki1(m, n, k, dA, m, dB, k, C, m, L)
        except ValueError:
            continue
        out.append(row(dist, k, "ozaki1", L * (L + 1) // 2, 7 * L - 2, metrics(torch, C, hi, lo, ab)))
    return out


def two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def run_complex(oz, torch, dist, k, mn, svals, seed, Ls=()):
    """ZGEMM rows: the double-double product assembled from the four real double-double
    products (Re = ArBr - AiBi, Im = ArBi + AiBr) and |A||B| = (|Ar|+|Ai|)(|Br|+|Bi|)"""
    import oz2
    m = n = mn
    parts = [generate(m, k, dist, seed * 1000 + 11 + k, True), generate(m, k, dist, seed * 1000 + 13 + k, True),
             generate(k, n, dist, seed * 1000 + 77 + k, False), generate(k, n, dist, seed * 1000 + 79 + k, False)]
    Ar, Ai, Br, Bi = (torch.from_numpy(x.ravel(order="F").copy()).cuda() for x in parts)

    def dd(X, Y):
        h = torch.empty(m * n, dtype=torch.float64, device="cuda")
        l, a = torch.empty_like(h), torch.empty_like(h)
        oz.dd_reference(m, n, k, X, m, Y, k, h, l, a)
        return h, l, a

    (h1, l1, a1), (h2, l2, a2), (h3, l3, a3), (h4, l4, a4) = dd(Ar, Br), dd(Ai, Bi), dd(Ar, Bi), dd(Ai, Br)
    s, e = two_sum(h1, -h2)
    re_t = e + (l1 - l2)
    re_h, re_l = two_sum(s, re_t)
    s, e = two_sum(h3, h4)
    im_t = e + (l3 + l4)
    im_h, im_l = two_sum(s, im_t)
    hi = torch.cat([re_h, im_h])
    lo = torch.cat([re_l, im_l])
    absab = (a1 + a2 + a3 + a4).repeat(2)
    A = torch.stack([Ar, Ai], dim=1).reshape(-1)  # interleaved complex, column-major
    B = torch.stack([Br, Bi], dim=1).reshape(-1)
    Az = torch.view_as_complex(A.view(k, m, 2))  # rows of the view: columns of A
    Bz = torch.view_as_complex(B.view(n, k, 2))
    Cz = torch.mm(Bz, Az).reshape(-1)  # C^T row-major = C column-major
    out = [row("z" + dist, k, "zgemm_gpu", 0, 53, metrics(torch, torch.cat([Cz.real, Cz.imag]), hi, lo, absab))]
    C = torch.empty(2 * m * n, dtype=torch.float64, device="cuda")
    for s in svals:
        try:
            tk = oz2.Ozaki2.precision_bits_complex(k, s)
        except ValueError:
            continue
        oz.zgemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, s)
        Cc = C.view(-1, 2)
        out.append(row("z" + dist, k, "ozaki2_3m", s, tk, metrics(torch, torch.cat([Cc[:, 0], Cc[:, 1]]), hi, lo,
                                                                     absab)))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--k", default="256,1024,4096,16384")
    ap.add_argument("--s", default="4-24")
    ap.add_argument("--L", default="4-9")
    ap.add_argument("--dist", default="urand,phi0.5,phi2,phi4")
    ap.add_argument("--mn", type=int, default=512)
    ap.add_argument("--complex", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    import torch
    import oz2
    oz = oz2.Ozaki2(torch.cuda.current_stream())
    print(CSV_HEADER, flush=True)
    lines = []
    for dist in a.dist.split(","):
        for k in parse_ints(a.k):
            run = run_complex if a.complex else run_real
            for line in run(oz, torch, dist, k, a.mn, parse_ints(a.s), a.seed, parse_ints(a.L)):
                print(line, flush=True)
                lines.append(line)
    oz.close()
    return lines


if __name__ == "__main__":
    sys.exit(0 if main() is not None else 1)
