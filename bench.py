#!/usr/bin/env python
"""Benchmark: emulated FP64 DGEMM (Ozaki Scheme II on the INT8 tensor cores) on B200.

Workload (one step): C = 1.5 A B - 0.5 C with m = n = k = 8192, op = N,N, ldc = m + 16,
A and B i.i.d. U[-1,1) FP64 (seeded, generated on the device), s = 16 moduli.
Metric: FP64-equivalent TFLOP/s = 2 m n k / t. Inputs are 512 MiB each, larger than the
126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W]            this implementation
  python bench.py --impl reference [--steps K --warmup W]    the reference's CPU path

Under torchrun every rank runs its own full problem (weak scaling, no collective on the data
path); value = all ranks' work / max over ranks of the device-timed region.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "os2-xe_b200"))

METRIC = "FP64-equiv TFLOP/s at DGEMM-level error: adaptive-s batched vs fixed-s, 1 B200"
UNIT = "TFLOP/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="oz2", choices=["oz2", "reference"])
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--s", type=int, default=16)
    ap.add_argument("--no-extras", action="store_true", help="skip the e2e, cuBLAS and CPU legs")
    return ap.parse_args()


def workload(a):
    n = a.size
    return {"workload": f"dgemm {n}x{n}x{n} op=NN s={a.s} alpha=1.5 beta=-0.5 ldc=m+16 U[-1,1)",
            "m": n, "n": n, "k": n, "s": a.s, "alpha": 1.5, "beta": -0.5, "ldc": n + 16,
            "l2": "inputs (8 n^2 bytes each) larger than the 126 MB L2; no flush"}


# ------------------------------------------------------------------ clocks during the timed region
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ CPU legs (reference / oracle)
def cpu_sample(a, steps, warmup):
    """The reference's own CPU path (oracle/_ref: src/ozaki2_gpu.hpp compiled for the host) on a
    512 x 512 x k slice of the workload, all host threads; the C oracle when it was not built."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle, Ref, ref_available
    threads = os.cpu_count() or 1
    m = n = min(512, a.size)
    k = a.size
    rng = np.random.default_rng(7)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    C = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    if ref_available():
        lib, kind = Ref(), "reference"
        run = lambda: lib.dgemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, m, a.s)
    else:
        lib, kind = Oracle(), "port"
        run = lambda: lib.dgemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, m, a.s)
    lib.set_threads(threads)
    for _ in range(warmup):
        run()
    t0 = time.perf_counter()
    for _ in range(steps):
        run()
    t = (time.perf_counter() - t0) / max(steps, 1)
    return {"value": 2.0 * m * n * k / t / 1e12, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"dgemm {m}x{n}x{k} op=NN s={a.s} (a {m}x{n} block of C at full k), "
                      f"{'src/ozaki2_gpu.hpp built for the host' if kind == 'reference' else 'C oracle'}",
            "seconds_per_step": t}


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    warm = min(a.warmup, 1)
    cb = cpu_sample(a, max(1, min(a.steps, 3)), warm)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": cb["seconds_per_step"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (int8 residues)",
            "data": "synthetic", "config": workload(a),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ this implementation
def launches_per_call(t):
    """kernels of liboz2 per emulated GEMM: 2 scale, split of B per column tile, split of A once
    (or per tile when there are several row tiles), k_chunks GEMMs and one CRT per tile"""
    tiles = t.pm * t.pn
    return 2 + t.pn + (tiles if t.pm > 1 else 1) + tiles * t.k_chunks + tiles


def grouped_leg(oz2, torch, dev, stream, reps=5):
    """512 DGEMMs, m, n, k log-uniform in [32, 2048], ops uniform over NN/NT/TN/TT, s uniform in
    14..20, U[-1,1): one grouped call (autotuned GEMM configuration, replayed from a CUDA graph)
    against 512 sequential calls of the same problems. FP64-equivalent TFLOP/s = sum 2 m n k / t."""
    import math
    import random
    rnd = random.Random(2024)
    g = torch.Generator(device=dev)
    g.manual_seed(77)
    probs, flops = [], 0.0
    for _ in range(512):
        m, n, k = (int(math.exp(rnd.uniform(math.log(32), math.log(2048)))) for _ in range(3))
        ta, tb = rnd.choice("NT"), rnd.choice("NT")
        s = rnd.randint(14, 20)
        lda, ldb = (m if ta == "N" else k), (k if tb == "N" else n)
        A = torch.rand(m * k, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        B = torch.rand(k * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        C = torch.zeros(m * n, dtype=torch.float64, device=dev)
        probs.append((ta, tb, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, m, s))
        flops += 2.0 * m * n * k
    oz = oz2.Ozaki2(stream)
    cfg = oz.autotune_grouped(probs)
    oz.set_graph_mode(True)
    oz.gemm_grouped(probs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        oz.gemm_grouped(probs)
    e1.record(stream)
    torch.cuda.synchronize()
    t_grouped = e0.elapsed_time(e1) / reps
    for p in probs:
        oz.gemm(*p)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        for p in probs:
            oz.gemm(*p)
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / reps
    oz.check_device_error()
    oz.close()
    return {"workload": "512 dgemm, m,n,k log-uniform [32,2048], ops uniform NN/NT/TN/TT, s uniform 14..20, "
                        "U[-1,1)", "grouped_tflops": flops / (t_grouped * 1e-3) / 1e12, "grouped_ms": t_grouped,
            "sequential_tflops": flops / (t_seq * 1e-3) / 1e12, "sequential_ms": t_seq,
            "speedup": t_seq / t_grouped, "gemm_config": cfg, "graph": True}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference_arm(a)
    import torch
    import torch.distributed as dist
    import oz2

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    n = a.size
    m = k = n
    ldc = m + 16
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    A = torch.rand(m * k, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    B = torch.rand(k * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C0 = torch.rand(ldc * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C = C0.clone()
    stream = torch.cuda.current_stream()
    oz = oz2.Ozaki2(stream)

    def step():
        oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, a.s)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    oz.check_device_error()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1) / a.steps
    oz.check_device_error()
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    flops = 2.0 * m * n * k
    value = world * flops / (ms * 1e-3) / 1e12

    # per-phase device times (CUDA events between phases, on the launching stream)
    oz.set_profiling(True)
    st_sum = [0.0, 0.0, 0.0, 0.0]
    for _ in range(a.steps):
        step()
        st = oz.stage_times()
        for i, v in enumerate((st.scale_ms, st.split_ms, st.gemm_ms, st.crt_ms)):
            st_sum[i] += v / a.steps
    oz.set_profiling(False)
    tiling = oz.last_tiling()
    gemm_ms = st_sum[2]
    pk = peaks()
    int8_ops = 2.0 * a.s * m * n * k
    achieved = int8_ops / (gemm_ms * 1e-3) / 1e12
    bf16 = pk.get("bf16_tflops")
    peak = 2.0 * bf16 if bf16 else 2.0 * 1590.0
    extras = {}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (int8 residues, int32 accumulate)", "data": "synthetic", "config": workload(a),
            "clocks": clk.summary(), "gpu_launches": launches_per_call(tiling) * a.steps,
            "stage_ms": {"scale": st_sum[0], "split": st_sum[1], "gemm": st_sum[2], "crt": st_sum[3]},
            "tiling": {"mb": tiling.mb, "nb": tiling.nb, "pm": tiling.pm, "pn": tiling.pn,
                       "k_chunks": tiling.k_chunks, "workspace_bytes": tiling.workspace_bytes},
            "roofline": {"bound": "tensor", "kernel": "gemm_i8_modm_kernel", "achieved": achieved, "peak": peak,
                         "unit": "TOPS (int8)", "frac": achieved / peak,
                         "peak_note": ("2 x measured dense bf16 (MEASURED_PEAKS.json bf16_tflops): B200 int8 "
                                       "dense rate is twice bf16" if bf16 else "2 x fallback bf16 1.59 PF"),
                         "algorithmic": "2 s m n k int8 ops per call", "traffic": None}}

    if not a.no_extras:
        # e2e through the public API with host buffers: H2D of A, B, C and D2H of C every step
        hA = torch.empty(m * k, dtype=torch.float64, pin_memory=True)
        hB = torch.empty(k * n, dtype=torch.float64, pin_memory=True)
        hC = torch.empty(ldc * n, dtype=torch.float64, pin_memory=True)
        hA.copy_(A)
        hB.copy_(B)
        hC.copy_(C0)
        dA, dB, dC = torch.empty_like(A), torch.empty_like(B), torch.empty_like(C0)
        out = torch.empty(ldc * n, dtype=torch.float64, pin_memory=True)

        def e2e_step():
            dA.copy_(hA, non_blocking=True)
            dB.copy_(hB, non_blocking=True)
            dC.copy_(hC, non_blocking=True)
            oz.gemm("N", "N", m, n, k, 1.5, dA, m, dB, k, -0.5, dC, ldc, a.s)
            out.copy_(dC, non_blocking=True)

        for _ in range(min(a.warmup, 2)):
            e2e_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / a.steps
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        line["e2e"] = {"value": world * flops / (e2e_ms * 1e-3) / 1e12, "unit": UNIT,
                       "h2d_bytes_per_step": 8 * (m * k + k * n + ldc * n), "d2h_bytes_per_step": 8 * ldc * n,
                       "ms_per_step": e2e_ms}
        del dA, dB, dC
        # native cuBLAS FP64 DGEMM on the same device, same shape (reference point, not the product)
        X = A.view(k, m).t()
        Y = B.view(n, k).t()
        torch.mm(X, Y)
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(3):
            torch.mm(X, Y)
        c1.record(stream)
        torch.cuda.synchronize()
        extras["cublas_dgemm_tflops"] = flops / (c0.elapsed_time(c1) / 3 * 1e-3) / 1e12
        # cuBLASLt int8 GEMM at the same shape, for context on the tensor-pipe peak
        try:
            Xi = torch.randint(-128, 127, (m, k), dtype=torch.int8, device=dev)
            Yi = torch.randint(-128, 127, (k, n), dtype=torch.int8, device=dev).t().contiguous().t()
            torch._int_mm(Xi, Yi)
            torch.cuda.synchronize()
            c0.record(stream)
            for _ in range(5):
                torch._int_mm(Xi, Yi)
            c1.record(stream)
            torch.cuda.synchronize()
            extras["cublaslt_int8_tops"] = 2.0 * m * n * k / (c0.elapsed_time(c1) / 5 * 1e-3) / 1e12
        except Exception as e:  # noqa: BLE001
            extras["cublaslt_int8_tops"] = f"unavailable: {type(e).__name__}"
        line["vs_cublas_dgemm"] = value / world / extras["cublas_dgemm_tflops"]
        extras["grouped_c4"] = grouped_leg(oz2, torch, dev, stream)
        if rank == 0:
            line["cpu_baseline"] = {k2: v for k2, v in cpu_sample(a, 1, 0).items() if k2 != "seconds_per_step"}
    line["extras"] = extras
    if rank == 0:
        print(json.dumps(line), flush=True)
    oz.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
