"""Training and loading of the MLP that picks the number of moduli s per C tile.

Labels come from the emulator itself: for a sample tile (512 x 512 x k, or an edge tile with
fewer rows or columns, of a problem with inputs (u - 0.5) exp(phi g), per-row / per-column
exponent offsets), the label is the smallest s whose result meets the DGEMM-level target, every
entry within k 2^-53 (|A||B|)_ij of the exact product, measured against the library's
double-double reference (oz2_dd_reference); 25 when no s <= 24 does (the MLP's last class: "more
than 24", which the library resolves with its arbiter, up to the extended sets' s = 32 or native
FP64). Features are the
library's own tile features (oz2_tile_features). Training runs the hand-written CUDA kernel
(oz2_mlp_train). The model is saved as JSON: parameters, decision threshold, tile, provenance.
"""
import json
import math
import os
import random

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "adaptive_mlp.json")
MODEL_VERSION = 1


def make_problem(torch, dev, m, n, k, phi, offsets, gen):
    """column-major A (m x k), B (k x n): (u - 0.5) exp(phi g), rows of A and columns of B scaled by
    2^U[-offsets, offsets] (integer exponents)"""
    def mat(rows, cols, row_scaled):
        u = torch.rand((cols, rows), dtype=torch.float64, device=dev, generator=gen) - 0.5
        g = torch.randn((cols, rows), dtype=torch.float64, device=dev, generator=gen)
        x = u * torch.exp(phi * g)
        if offsets:
            if row_scaled:  # per row of the column-major matrix
                e = torch.randint(-offsets, offsets + 1, (1, rows), device=dev, generator=gen).double()
            else:  # per column
                e = torch.randint(-offsets, offsets + 1, (cols, 1), device=dev, generator=gen).double()
            x = x * torch.exp2(e)
        return x.contiguous().view(-1)  # (cols, rows) row-major = (rows, cols) column-major
    return mat(m, k, True), mat(k, n, False)


def label_tile(oz, torch, A, B, m, n, k, target_bits=53, smin=2, smax=24):
    """smallest s in [smin, smax] meeting the target on C = A B (N, N); smax + 1 (native FP64)
    when none does"""
    import oz2
    dev = A.device
    hi = torch.empty(m * n, dtype=torch.float64, device=dev)
    lo = torch.empty_like(hi)
    ab = torch.empty_like(hi)
    oz.dd_reference(m, n, k, A, m, B, k, hi, lo, ab)
    C = torch.empty(m * n, dtype=torch.float64, device=dev)

    def ok(s):
        try:
            oz.gemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m, s)
        except ValueError:  # s too small for k
            return False
        return oz.error_ratio(m, n, k, C, m, hi, lo, ab, target_bits) <= 1.0

    lo_s, hi_s = smin, smax
    if not ok(hi_s):
        return smax + 1
    while lo_s < hi_s:
        mid = (lo_s + hi_s) // 2
        if ok(mid):
            hi_s = mid
        else:
            lo_s = mid + 1
    return lo_s


def generate_dataset(oz, count, seed=1, tile=512, k_range=(256, 4096), phi_range=(0.0, 8.0), offsets=40,
                     target_bits=53, edge_fraction=0.3):
    """features (float32 [count, F]), labels (int32 [count]) and analytic s (int32 [count]) on
    the device"""
    import torch
    dev = torch.device("cuda")
    rnd = random.Random(seed)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    feats, labels, s_an = [], [], []
    for _ in range(count):
        k = int(math.exp(rnd.uniform(math.log(k_range[0]), math.log(k_range[1]))))
        phi = rnd.uniform(*phi_range)
        # edge tiles of a problem hold fewer rows or columns
        mt = tile if rnd.random() >= edge_fraction else rnd.randint(1, tile)
        nt = tile if rnd.random() >= edge_fraction else rnd.randint(1, tile)
        A, B = make_problem(torch, dev, mt, nt, k, phi, offsets, gen)
        C = torch.zeros(mt * nt, dtype=torch.float64, device=dev)
        f, sa = oz.tile_features([("N", "N", mt, nt, k, 1.0, A, mt, B, k, 0.0, C, mt, 16)], target_bits)
        feats.append(f[0])
        s_an.append(sa[0])
        labels.append(label_tile(oz, torch, A, B, mt, nt, k, target_bits))
    return (torch.stack(feats), torch.tensor(labels, dtype=torch.int32, device=dev),
            torch.stack(s_an).to(torch.int32))


def init_params(seed=0):
    """Xavier-uniform weights, zero biases, in the library's parameter layout"""
    import oz2
    info = oz2.mlp_info()
    F, H, Cn = info["features"], info["hidden"], info["classes"]
    rnd = random.Random(seed)

    def block(fan_out, fan_in):
        a = math.sqrt(6.0 / (fan_in + fan_out))
        return [rnd.uniform(-a, a) for _ in range(fan_out * fan_in)] + [0.0] * fan_out
    params = block(H, F) + block(H, H) + block(Cn, H)
    assert len(params) == info["params"]
    return params


THRESHOLDS = (0.5, 0.8, 0.9, 0.95, 0.98, 0.99, 0.995, 0.999, 0.9995, 0.9999)
NATIVE_COST = 36.0  # a native FP64 tile costs about as much as 36 moduli of emulation


def tile_cost(s):
    return NATIVE_COST if s > 32 else float(s)


def evaluate(oz, params, feats, labels, s_an, thresholds=THRESHOLDS):
    """per threshold, with s = min(MLP s, analytic s) as the library runs it: exact-label rate,
    under-prediction rate (tiles the probe must catch), mean s, native fraction, and the expected
    cost per tile in moduli (a native tile counting NATIVE_COST) when every under-predicted tile
    is rerun at its analytic s"""
    out = {}
    lab = labels.cpu().tolist()
    an = s_an.cpu().tolist()
    n = len(lab)
    for th in thresholds:
        s = [min(a, b) for a, b in zip(oz.mlp_infer(params, feats, th).cpu().tolist(), an)]
        under = [a < b for a, b in zip(s, lab)]
        cost = sum(tile_cost(v) for v in s) + sum(tile_cost(a) for a, u in zip(an, under) if u)
        out[str(th)] = {"exact": sum(a == b for a, b in zip(s, lab)) / n, "under": sum(under) / n,
                        "mean_s": sum(s) / n, "mean_label": sum(lab) / n, "mean_analytic": sum(an) / n,
                        "native": sum(v > 24 for v in s) / n, "native_label": sum(v > 24 for v in lab) / n,
                        "expected_cost": cost / n,
                        "label_cost": sum(tile_cost(v) for v in lab) / n,
                        "analytic_cost": sum(tile_cost(v) for v in an) / n}
    return out


def save_model(path, params, threshold, tile=512, info=None):
    with open(path, "w") as f:
        json.dump({"version": MODEL_VERSION, "tile": tile, "threshold": threshold, "params": params,
                   "info": info or {}}, f)


def load_model(path=None):
    with open(path or DEFAULT_MODEL) as f:
        model = json.load(f)
    if model.get("version") != MODEL_VERSION:
        raise ValueError(f"unsupported model version {model.get('version')}")
    return model


def train_default(out_path=DEFAULT_MODEL, n_train=6000, n_val=2000, epochs=600, lr=3e-3, seed=7, max_under=0.0):
    """generates labels, trains, and picks the threshold with the fewest expected moduli per tile
    (reruns counted) among those whose validation under-prediction rate is at most max_under: the
    probe checks a few columns of a tile only, so the MLP itself must rarely choose too few"""
    import torch
    import oz2
    oz = oz2.Ozaki2(torch.cuda.current_stream())
    ftr, ltr, _ = generate_dataset(oz, n_train, seed=seed)
    fva, lva, ava = generate_dataset(oz, n_val, seed=seed + 1000)
    params, losses = oz.mlp_train(ftr, ltr, init_params(seed), epochs=epochs, lr=lr, seed=seed)
    ev = evaluate(oz, params, fva, lva, ava)
    ok = [th for th in ev if ev[th]["under"] <= max_under] or [max(ev, key=float)]
    threshold = float(min(ok, key=lambda th: ev[th]["expected_cost"]))
    info = {"n_train": n_train, "n_val": n_val, "epochs": epochs, "lr": lr, "seed": seed,
            "loss_first": losses[0], "loss_last": losses[-1], "validation": ev,
            "train_label_hist": torch.bincount(ltr.long(), minlength=26).cpu().tolist()}
    save_model(out_path, params, threshold, info=info)
    oz.close()
    return info


if __name__ == "__main__":
    import sys
    print(json.dumps(train_default(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_MODEL), indent=1))
