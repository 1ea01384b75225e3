#!/usr/bin/env python
"""Benchmark: emulated FP64 DGEMM (Ozaki Scheme II on the INT8 tensor cores) on B200.

Headline workload: the adaptive-s stream of 10,000 DGEMMs with m = n = k log-uniform in
[256, 4096], inputs (u - 0.5) exp(phi g) with u ~ U[0,1), g ~ N(0,1), phi per problem uniform in
[0, 8], the rows of A and the columns of B scaled by 2^e, e uniform in [-40, 40]; alpha = 1,
beta = 0, target DGEMM-level error (|C - AB| <= k 2^-53 (|A||B|)_ij). The stream is cut into
`--steps` batches; one step = one batched adaptive call over one batch (10,000 / steps problems,
at most 512), generated on the device with a seeded generator before the step and timed alone
with CUDA events, so every timed problem is distinct; each batch (tens of GB) is far larger than
the 126 MB L2. s is chosen per 512 x 512 tile: certified where a tile needs 23 or more moduli by
the analytic rule, else by the MLP (probed, rerun at the arbiter's s on failure); tiles no s <= 24
serves run in native FP64. Metric: FP64-equivalent TFLOP/s = sum 2 m n k / t. The fixed-s forms
of the same batches (per-problem analytic s batched and as plain calls, the certified per-problem
s, cuBLAS DGEMM for everything, s = 24, the reference's moduli_for_bits(k, 53)) are timed step by
step on the same problems, and every output of every form is checked against a double-double
product. Extras: the m = n = k = 8192 DGEMM at s = 16 (alpha 1.5, beta -0.5, ldc = m + 16)
against cuBLAS DGEMM, the ZGEMM 4096^3, and the grouped launch of 512 uneven DGEMMs.

  python bench.py [--gpus N --steps K --warmup W]            this implementation
  python bench.py --impl reference [--steps K --warmup W]    the reference's CPU path

Under torchrun every rank runs its own stream (weak scaling, no collective on the data path);
value = all ranks' work / the sum over steps of the slowest rank's step time.
"""
import argparse
import gc
import json
import math
import os
import random
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "os2-xe_b200"))

METRIC = "FP64-equiv TFLOP/s at DGEMM-level error: adaptive-s batched vs fixed-s, 1 B200"
UNIT = "TFLOP/s"
TARGET_BITS = 53
MAX_BATCH = 512          # problems per step: inputs, outputs and the check's references of a batch
WORKSPACE = 24 << 30     # workspace limit of the bench's handle (the same for every form)
E2E_BATCH = 64           # problems per step of the end-to-end leg (pinned host arenas)
# DRAM bytes / algorithmic bytes of the residue GEMM on this stream, from one ncu capture of a
# small case (profiles/gemm_i8_modm_kernel_traffic_adaptive_stream.md): 44.35 GB over 44.37 GB
GEMM_TRAFFIC_RATIO = 0.9994


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="oz2", choices=["oz2", "reference"])
    ap.add_argument("--problems", type=int, default=10000, help="problems of the adaptive-s stream")
    ap.add_argument("--batch", type=int, default=0,
                    help="problems per step (default: problems / steps, at most %d)" % MAX_BATCH)
    ap.add_argument("--forms", default="all", help="'all' or 'headline': the fixed-s forms beside the headline")
    ap.add_argument("--probe-study", action="store_true",
                    help="instead of the bench line: problems over the bound per MLP threshold and probe kind")
    ap.add_argument("--seed", type=int, default=2025)
    ap.add_argument("--size", type=int, default=8192, help="m = n = k of the DGEMM extra")
    ap.add_argument("--s", type=int, default=16, help="moduli of the DGEMM extra")
    ap.add_argument("--k", type=int, default=0, help="inner dimension of the DGEMM extra (default: --size)")
    ap.add_argument("--no-extras", action="store_true", help="skip the DGEMM, grouped and CPU legs")
    ap.add_argument("--split-kernel", type=int, default=0, choices=(0, 1),
                    help="real split kernel: 0 integer pipe (dp4a, default), 1 tensor core")
    ap.add_argument("--crt-kernel", type=int, default=2, choices=(0, 1, 2),
                    help="real CRT kernel: 2 auto (default: tensor core for 7- and 8-limb plans), 1 tensor core, 0 dp2a")
    ap.add_argument("--scale-fusion", type=int, default=0, choices=(0, 1),
                    help="scale pass fused into the split for k <= 2048 (1) or separate (0, default)")
    ap.add_argument("--crt-fusion", type=int, default=0, choices=(0, 1),
                    help="CRT in the GEMM epilogue for s <= 8 (1) or a separate CRT launch (0, default)")
    ap.add_argument("--probe-kind", type=int, default=-1, choices=(-1, 0, 1, 2, 3),
                    help="probe of the MLP tiles: -1 the library default, 0 columns, 1 Freivalds, 2 both, 3 none")
    ap.add_argument("--dgemm-only", action="store_true",
                    help="time only the DGEMM of --size and --s (a profiling aid; not the headline)")
    return ap.parse_args()


def batch_size(a):
    return a.batch or max(1, min(MAX_BATCH, -(-a.problems // a.steps)))


def workload(a):
    b = batch_size(a)
    timed = min(a.problems, b * a.steps)
    return {"workload": f"adaptive-s stream of {a.problems} dgemm (the first {timed} timed, {b} per step, each "
                        "batch generated before its step), m=n=k log-uniform [256,4096], (u-0.5)exp(phi g), "
                        "phi~U[0,8] per problem, rows of A / columns of B scaled by 2^U[-40,40], alpha=1 beta=0, "
                        "target 53 bits, s per 512x512 tile",
            "problems": a.problems, "problems_timed": timed, "batch": b, "tile": 512, "target_bits": TARGET_BITS,
            "seed": a.seed, "l2": "each batch holds tens of GB, far larger than the 126 MB L2; no flush"}


def stream_specs(seed, count):
    """(n, phi, seed) of the first `count` problems of the stream"""
    rnd = random.Random(seed)
    out = []
    for i in range(count):
        n = int(math.exp(rnd.uniform(math.log(256), math.log(4096))))
        phi = rnd.uniform(0.0, 8.0)
        out.append((n, phi, seed * 1000003 + i))
    return out


def make_problem(torch, dev, n, phi, seed):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)

    def mat(row_scaled):
        x = torch.rand((n, n), dtype=torch.float64, device=dev, generator=g) - 0.5  # [col][row]
        x *= torch.exp(phi * torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))
        e = torch.randint(-40, 41, (1, n) if row_scaled else (n, 1), device=dev, generator=g).double()
        return (x * torch.exp2(e)).view(-1)
    A = mat(True)    # column-major n x n, rows scaled
    B = mat(False)   # column-major n x n, columns scaled
    C = torch.zeros(n * n, dtype=torch.float64, device=dev)
    return {"n": n, "phi": phi, "A": A, "B": B, "C": C}


def as_args(p, s=16, C_=None):
    n = p["n"]
    return ("N", "N", n, n, n, 1.0, p["A"], n, p["B"], n, 0.0, p["C"] if C_ is None else C_, n, s)


def flops_of(batch):
    return sum(2.0 * p["n"] ** 3 for p in batch)


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
                                          "-lms", "50", "-i", str(self.index)], stdout=subprocess.PIPE,
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
def host_problem(n, phi, seed):
    """one problem of the stream generated by numpy (same distribution as the device generator,
    not the same numbers): column-major A and B"""
    import numpy as np
    rng = np.random.default_rng(seed)
    A = (rng.random((n, n)) - 0.5) * np.exp(phi * rng.standard_normal((n, n)))
    A = np.asfortranarray(A * np.ldexp(1.0, rng.integers(-40, 41, (n, 1))))
    B = (rng.random((n, n)) - 0.5) * np.exp(phi * rng.standard_normal((n, n)))
    B = np.asfortranarray(B * np.ldexp(1.0, rng.integers(-40, 41, (1, n))))
    return A, B


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        return max((d.get("num_threads", 0) for d in threadpool_info() if d.get("user_api") == "blas"), default=0)
    except Exception:  # noqa: BLE001
        return 0


class CpuStream:
    """The reference's own CPU path (oracle/_ref: src/ozaki2_gpu.hpp built for the host, all host
    threads; the C oracle where it was not built) over the stream's problems in stream order, each
    at its per-problem analytic s (the fixed s that meets the target). The reference's Ozaki2::gemm
    takes s <= 24 only (make_plan rejects more, src/ozaki2_gpu.hpp:160-161), so a problem whose
    analytic s is 25 runs as host FP64 DGEMM (numpy's BLAS, the reference bench's --cpu path,
    benchmarks/bench_ozaki2.cpp:133-142), and its time counts. Every call's status is checked."""

    def __init__(self, a):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import adaptive_oracle
        from pyoracle import Oracle, Ref, ref_available
        self.ao = adaptive_oracle
        self.threads = os.cpu_count() or 1
        self.is_ref = ref_available()
        self.lib = Ref() if self.is_ref else Oracle()
        self.kind = "reference" if self.is_ref else "port"
        self.lib.set_threads(self.threads)
        self.plans = Oracle()
        self.specs = stream_specs(a.seed, a.problems)
        self.pos = 0
        self.native = self.emulated = 0

    def step(self, budget_s):
        """problems from the current position until budget_s seconds of compute: (flops, seconds)"""
        import numpy as np
        flops = secs = 0.0
        while secs < budget_s and self.pos < len(self.specs):
            n, phi, seed = self.specs[self.pos]
            self.pos += 1
            A, B = host_problem(n, phi, seed)
            C = np.zeros((n, n), order="F")
            sv = self.ao.problem_analytic_s(self.plans, "N", "N", n, n, n, A, B, TARGET_BITS)
            t0 = time.perf_counter()
            if sv > 24:
                np.matmul(A, B, out=C)
                self.native += 1
            else:
                st = self.lib.dgemm("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, sv)
                st = st[0] if isinstance(st, tuple) else st
                if st != 0:
                    raise RuntimeError(f"CPU path failed on problem {self.pos - 1} (n={n}, s={sv}): status {st}")
                self.emulated += 1
            secs += time.perf_counter() - t0
            flops += 2.0 * n ** 3
        return flops, secs

    def describe(self, problems, secs):
        what = "src/ozaki2_gpu.hpp built for the host" if self.is_ref else "the C oracle"
        return (f"{problems} problems of the same stream in stream order (numpy-generated, same distribution), "
                f"{self.emulated} at their per-problem analytic s through {what}, {self.native} whose analytic s "
                f"exceeds 24 as host FP64 DGEMM (numpy BLAS); {secs:.1f} s of compute, {self.threads} threads")


def cpu_sample(a, budget_s=12.0):
    cs = CpuStream(a)
    flops, secs = cs.step(budget_s)
    return {"value": flops / secs / 1e12, "unit": UNIT, "cores": cs.threads, "kind": cs.kind,
            "sample": cs.describe(cs.pos, secs)}


def cpu_dgemm_sample(a, budget_s=8.0):
    """host FP64 DGEMM (numpy's BLAS, all its threads) over the stream's problems in stream order:
    the reference bench's --cpu baseline (benchmarks/bench_ozaki2.cpp:133-142). DGEMM-level error
    by construction."""
    import numpy as np
    flops = secs = 0.0
    done = 0
    for n, phi, seed in stream_specs(a.seed, a.problems):
        if secs >= budget_s:
            break
        A, B = host_problem(n, phi, seed)
        C = np.empty((n, n), order="F")
        np.matmul(A, B, out=C)  # warm (BLAS threads, pages)
        t0 = time.perf_counter()
        np.matmul(A, B, out=C)
        secs += time.perf_counter() - t0
        flops += 2.0 * n ** 3
        done += 1
    threads = blas_threads()
    return {"value": flops / secs / 1e12, "unit": UNIT, "cores": threads or (os.cpu_count() or 1),
            "kind": "host fp64 dgemm",
            "sample": f"the first {done} problems of the same stream (numpy-generated), numpy.matmul FP64 "
                      f"(OpenBLAS, {threads or 'all'} threads), {secs:.1f} s of compute"}


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cs = CpuStream(a)
    for _ in range(a.warmup):
        cs.step(0.5)
    first = cs.pos
    cs.emulated = cs.native = 0  # the description counts the timed problems only
    flops = secs = 0.0
    for _ in range(a.steps):
        f, t = cs.step(4.0)
        flops, secs = flops + f, secs + t
    value = flops / secs / 1e12
    sample = cs.describe(cs.pos - first, secs) + "; about 4 s of compute per step"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": secs / a.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (int8 residues)",
            "data": "synthetic", "config": workload(a),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cs.threads, "kind": cs.kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ this implementation
def launches_per_call(t):
    """kernels of liboz2 per emulated GEMM: 2 scale, split of B per column tile, split of A once
    (or per tile when there are several row tiles), k_chunks GEMMs and one CRT per tile"""
    tiles = t.pm * t.pn
    return 2 + t.pn + (tiles if t.pm > 1 else 1) + tiles * t.k_chunks + tiles


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def int8_peak():
    bf16 = peaks().get("bf16_tflops")
    if bf16:
        return 2.0 * bf16, ("2 x measured dense bf16 (MEASURED_PEAKS.json bf16_tflops): B200 int8 dense rate is "
                            "twice bf16")
    return 2.0 * 1590.0, "2 x fallback bf16 1.59 PF"


class NoGC:
    """Python's cyclic garbage collector off inside a timed region, as timeit does: a collection
    there stalls the host thread that issues the launches (tens to hundreds of ms in a process
    holding this many objects); it runs at the next allocation after the region instead"""

    def __enter__(self):
        self.was = gc.isenabled()
        gc.disable()
        return self

    def __exit__(self, *exc):
        if self.was:
            gc.enable()


class Timer:
    """CUDA events on the launching stream around a region (garbage collector off)"""

    def __init__(self, torch, stream):
        self.torch, self.stream = torch, stream
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def __enter__(self):
        self.nogc = NoGC().__enter__()
        self.torch.cuda.synchronize()
        self.e0.record(self.stream)
        return self

    def __exit__(self, *exc):
        self.e1.record(self.stream)
        self.torch.cuda.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)
        self.nogc.__exit__()


def sharded_leg(a, oz2, torch, dev, stream, dist, world, rank):
    """One DGEMM m = n = k = 8192, s = 16, alpha 1.5, beta -0.5, U[-1,1), split over the ranks as
    C blocks (strong scaling, oz2.sharded): every rank holds the same A, B and C (one seed), times
    its block (CUDA events, max over ranks), then the all-gather of the blocks, and checks the
    gathered C against its own unsharded call bit for bit (mismatches summed over ranks)."""
    from oz2 import sharded
    n = a.size
    m = k = n
    g = torch.Generator(device=dev)
    g.manual_seed(4321)
    A = torch.rand(m * k, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    B = torch.rand(k * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C0 = torch.rand(m * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C = C0.clone()
    oz = oz2.Ozaki2(stream)
    sho = sharded.ShardedOzaki2(oz)
    reps = 10

    def local():
        C.copy_(C0)
        sho.local_gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, m, a.s)

    for _ in range(3):
        local()
    with Timer(torch, stream) as t:
        for _ in range(reps):
            local()
    copy_ms = 0.0
    with Timer(torch, stream) as tc:
        for _ in range(reps):
            C.copy_(C0)
    copy_ms = tc.ms / reps
    ms_local = max(t.ms / reps - copy_ms, 1e-6)
    dist.barrier()
    with Timer(torch, stream) as tg:
        sho.gather(C, m, m, n)
    ms_gather = tg.ms
    full = C0.clone()
    oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, full, m, a.s)
    torch.cuda.synchronize()
    bad = torch.tensor([float((C.view(torch.int64) != full.view(torch.int64)).sum().item())], device=dev)
    dist.all_reduce(bad, op=dist.ReduceOp.SUM)
    ms_l, _ = over_ranks(dist, torch, world, dev, ms_local, 0.0)
    ms_g, _ = over_ranks(dist, torch, world, dev, ms_gather, 0.0)
    (r0, r1), (c0, c1) = sho.block(m, n)
    oz.close()
    del A, B, C0, C, full
    torch.cuda.empty_cache()
    flops = 2.0 * m * n * k
    return {"workload": f"dgemm {n}x{n}x{n} op=NN s={a.s} alpha=1.5 beta=-0.5 U[-1,1), C blocks over {world} ranks",
            "grid": list(sharded.grid_shape(world, m, n)), "rank0_block": [[r0, r1], [c0, c1]],
            "scaling": "strong", "ms_block_max": ms_l, "tflops_blocks": flops / (ms_l * 1e-3) / 1e12,
            "ms_gather": ms_g, "tflops_with_gather": flops / ((ms_l + ms_g) * 1e-3) / 1e12,
            "entries_differing_from_unsharded": int(bad.item())}


def grouped_leg(oz2, torch, dev, stream, reps=5):
    """512 DGEMMs, m, n, k log-uniform in [32, 2048], ops uniform over NN/NT/TN/TT, s uniform in
    14..20, U[-1,1): one grouped call (autotuned GEMM configuration, replayed from a CUDA graph)
    against 512 sequential calls of the same problems. FP64-equivalent TFLOP/s = sum 2 m n k / t."""
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
    with Timer(torch, stream) as tg:
        for _ in range(reps):
            oz.gemm_grouped(probs)
    for p in probs:
        oz.gemm(*p)
    with Timer(torch, stream) as ts:
        for _ in range(reps):
            for p in probs:
                oz.gemm(*p)
    oz.check_device_error()
    oz.close()
    t_grouped, t_seq = tg.ms / reps, ts.ms / reps
    return {"workload": "512 dgemm, m,n,k log-uniform [32,2048], ops uniform NN/NT/TN/TT, s uniform 14..20, "
                        "U[-1,1)", "grouped_tflops": flops / (t_grouped * 1e-3) / 1e12, "grouped_ms": t_grouped,
            "sequential_tflops": flops / (t_seq * 1e-3) / 1e12, "sequential_ms": t_seq,
            "speedup": t_seq / t_grouped, "gemm_config": cfg, "graph": True}


def dgemm_leg(a, oz2, torch, dev, stream, rank):
    """m = n = k = 8192 DGEMM at s = 16, alpha 1.5, beta -0.5, ldc = m + 16, U[-1,1): device time,
    stage times, the GEMM kernel against the int8 roofline, end to end with host buffers, and
    native cuBLAS DGEMM / cuBLASLt int8 at the same shape."""
    n = a.size
    m = n
    k = a.k or n
    ldc = m + 16
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    A = torch.rand(m * k, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    B = torch.rand(k * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C0 = torch.rand(ldc * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C = C0.clone()
    oz = oz2.Ozaki2(stream)
    steps = 20

    def step():
        oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, a.s)

    for _ in range(3):
        step()
    with Timer(torch, stream) as t:
        for _ in range(steps):
            step()
    ms = t.ms / steps
    flops = 2.0 * m * n * k
    oz.set_profiling(True)
    st_sum = [0.0] * 4
    for _ in range(steps):
        step()
        st = oz.stage_times()
        for i, v in enumerate((st.scale_ms, st.split_ms, st.gemm_ms, st.crt_ms)):
            st_sum[i] += v / steps
    oz.set_profiling(False)
    tiling = oz.last_tiling()
    peak, note = int8_peak()
    achieved = 2.0 * a.s * m * n * k / (st_sum[2] * 1e-3) / 1e12
    # accuracy of the product on a 1024 x 1024 block (full k) against a double-double product
    blk = min(1024, n)
    C2 = torch.empty(m * n, dtype=torch.float64, device=dev)
    oz.gemm("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C2, m, a.s)
    hi = torch.empty(blk * blk, dtype=torch.float64, device=dev)
    lo, ab = torch.empty_like(hi), torch.empty_like(hi)
    oz.dd_reference(blk, blk, k, A, m, B, k, hi, lo, ab)
    ulp, cr = oz.accuracy(blk, blk, C2, m, hi, lo)
    ratio = oz.error_ratio(blk, blk, k, C2, m, hi, lo, ab, TARGET_BITS)
    del C2, hi, lo, ab
    out = {"workload": f"dgemm {m}x{n}x{k} op=NN s={a.s} alpha=1.5 beta=-0.5 ldc=m+16 U[-1,1)",
           "accuracy": {"block": f"C[0:{blk}, 0:{blk}] of A B (alpha 1, beta 0) against double-double",
                        "ulp_max": ulp, "cr_frac": cr / (blk * blk), "dgemm_level_ratio": ratio},
           "tflops": flops / (ms * 1e-3) / 1e12, "ms": ms, "steps": steps,
           "stage_ms": {"scale": st_sum[0], "split": st_sum[1], "gemm": st_sum[2], "crt": st_sum[3]},
           "gpu_launches_per_call": launches_per_call(tiling),
           "roofline": {"bound": "tensor", "kernel": "gemm_i8_modm_kernel", "achieved": achieved, "peak": peak,
                        "unit": "TOPS (int8)", "frac": achieved / peak, "peak_note": note,
                        "algorithmic": "2 s m n k int8 ops per call"}}
    # the bandwidth-side stages against the measured copy bandwidth (algorithmic bytes per call:
    # scale 8 (mk + kn); split (8 + s)(mk + kn); CRT s mn residue bytes + 8 mn for C out + 8 mn in,
    # beta != 0)
    hbm = peaks().get("hbm_gbs") or 6650.0
    stage_bytes = {"scale": 8.0 * (m * k + k * n), "split": (8.0 + a.s) * (m * k + k * n),
                   "crt": (a.s + 16.0) * m * n}
    out["stage_roofline"] = {
        name: {"bound": "hbm", "algorithmic_bytes": b, "achieved_gbs": b / (st_sum[i] * 1e-3) / 1e9,
               "peak_gbs": hbm, "frac": b / (st_sum[i] * 1e-3) / 1e9 / hbm}
        for i, (name, b) in ((0, ("scale", stage_bytes["scale"])), (1, ("split", stage_bytes["split"])),
                             (3, ("crt", stage_bytes["crt"])))}
    out["stage_roofline_note"] = "peak: hbm_gbs of MEASURED_PEAKS.json (copy bandwidth); stage times as stage_ms"
    # the other op pairs at the same shape and s (alpha 1.5, beta -0.5)
    by_op = {}
    for ta, tb in (("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")):
        lda_, ldb_ = (m if ta == "N" else k), (k if tb == "N" else n)
        oz.gemm(ta, tb, m, n, k, 1.5, A, lda_, B, ldb_, -0.5, C, ldc, a.s)
        with Timer(torch, stream) as t:
            for _ in range(5):
                oz.gemm(ta, tb, m, n, k, 1.5, A, lda_, B, ldb_, -0.5, C, ldc, a.s)
        by_op[ta + tb] = flops / (t.ms / 5 * 1e-3) / 1e12
    out["tflops_by_op"] = by_op
    # end to end with host buffers: H2D of A, B, C and D2H of C every step
    hA = torch.empty(m * k, dtype=torch.float64, pin_memory=True)
    hB = torch.empty(k * n, dtype=torch.float64, pin_memory=True)
    hC = torch.empty(ldc * n, dtype=torch.float64, pin_memory=True)
    hA.copy_(A)
    hB.copy_(B)
    hC.copy_(C0)
    res = torch.empty(ldc * n, dtype=torch.float64, pin_memory=True)

    def e2e_step():
        A.copy_(hA, non_blocking=True)
        B.copy_(hB, non_blocking=True)
        C.copy_(hC, non_blocking=True)
        oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, a.s)
        res.copy_(C, non_blocking=True)

    e2e_step()
    with Timer(torch, stream) as t:
        for _ in range(5):
            e2e_step()
    out["e2e_tflops"] = flops / (t.ms / 5 * 1e-3) / 1e12
    # native cuBLAS FP64 DGEMM on the same device, same shape (reference point, not the product)
    X = A.view(k, m).t()
    Y = B.view(n, k).t()
    torch.mm(X, Y)
    with Timer(torch, stream) as t:
        for _ in range(3):
            torch.mm(X, Y)
    out["cublas_dgemm_tflops"] = flops / (t.ms / 3 * 1e-3) / 1e12
    out["vs_cublas_dgemm"] = out["tflops"] / out["cublas_dgemm_tflops"]
    try:
        Xi = torch.randint(-128, 127, (m, k), dtype=torch.int8, device=dev)
        Yi = torch.randint(-128, 127, (k, n), dtype=torch.int8, device=dev).t().contiguous().t()
        torch._int_mm(Xi, Yi)
        with Timer(torch, stream) as t:
            for _ in range(5):
                torch._int_mm(Xi, Yi)
        out["cublaslt_int8_tops"] = 2.0 * m * n * k / (t.ms / 5 * 1e-3) / 1e12
    except Exception as e:  # noqa: BLE001
        out["cublaslt_int8_tops"] = f"unavailable: {type(e).__name__}"
    # the other moduli counts of the same shape (alpha 1.5, beta -0.5), NN
    sweep = {}
    for sv in (8, 12, 16, 20, 24):
        oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, sv)
        with Timer(torch, stream) as t:
            for _ in range(5):
                oz.gemm("N", "N", m, n, k, 1.5, A, m, B, k, -0.5, C, ldc, sv)
        sweep[str(sv)] = flops / (t.ms / 5 * 1e-3) / 1e12
    out["tflops_by_s"] = sweep
    # the other DGEMM shapes of the workload table: 1024^3 at s = 16, and the k-split case
    # 1024 x 1024 x 262144 at s = 16 (three exact int32 chunks of k), NN, alpha 1, beta 0
    shapes = {}
    for name, (mm, nn, kk) in (("1024x1024x1024", (1024, 1024, 1024)), ("1024x1024x262144", (1024, 1024, 262144))):
        As = torch.rand(mm * kk, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        Bs = torch.rand(kk * nn, dtype=torch.float64, device=dev, generator=g) * 2 - 1
        Cs = torch.empty(mm * nn, dtype=torch.float64, device=dev)
        oz.gemm("N", "N", mm, nn, kk, 1.0, As, mm, Bs, kk, 0.0, Cs, mm, 16)
        with Timer(torch, stream) as t:
            for _ in range(5):
                oz.gemm("N", "N", mm, nn, kk, 1.0, As, mm, Bs, kk, 0.0, Cs, mm, 16)
        shapes[name] = {"s": 16, "tflops": 2.0 * mm * nn * kk / (t.ms / 5 * 1e-3) / 1e12, "ms": t.ms / 5,
                        "k_chunks": oz.last_tiling().k_chunks,
                        "l2": "inputs fit in L2 (warm)" if 8 * (mm * kk + kk * nn) < 100e6 else "inputs larger than L2"}
        del As, Bs, Cs
    out["other_shapes"] = shapes
    oz.check_device_error()
    oz.close()
    return out


def zgemm_leg(oz2, torch, dev, stream, rank):
    """ZGEMM 4096^3, op(A) = C, op(B) = N, alpha (1, 0.5), beta (0.25, -1), ldc = m + 8, s = 16,
    U[-1,1) real and imaginary parts: FP64-equivalent 8 m n k / t, against cuBLAS ZGEMM"""
    m = n = k = 4096
    ldc = m + 8
    g = torch.Generator(device=dev)
    g.manual_seed(4321 + rank)
    A = torch.rand(2 * k * m, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    B = torch.rand(2 * k * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    C = torch.rand(2 * ldc * n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    oz = oz2.Ozaki2(stream)
    for _ in range(2):
        oz.zgemm("C", "N", m, n, k, 1 + 0.5j, A, k, B, k, 0.25 - 1j, C, ldc, 16)
    with Timer(torch, stream) as t:
        for _ in range(5):
            oz.zgemm("C", "N", m, n, k, 1 + 0.5j, A, k, B, k, 0.25 - 1j, C, ldc, 16)
    ms = t.ms / 5
    oz.set_profiling(True)
    oz.zgemm("C", "N", m, n, k, 1 + 0.5j, A, k, B, k, 0.25 - 1j, C, ldc, 16)
    st = oz.stage_times()
    oz.set_profiling(False)
    oz.check_device_error()
    oz.close()
    flops = 8.0 * m * n * k
    Az = torch.view_as_complex(A.view(m, k, 2))  # row i of this view is column i of the stored A
    Bz = torch.view_as_complex(B.view(n, k, 2))
    # C^T = B^T conj(A) in row-major views of the column-major data
    torch.mm(Bz, Az.conj().t())
    with Timer(torch, stream) as t:
        for _ in range(3):
            torch.mm(Bz, Az.conj().t())
    zref = flops / (t.ms / 3 * 1e-3) / 1e12
    return {"workload": "zgemm 4096x4096x4096 op=(C,N) alpha=(1,0.5) beta=(0.25,-1) ldc=m+8 s=16 U[-1,1)",
            "tflops": flops / (ms * 1e-3) / 1e12, "ms": ms,
            "stage_ms": {"scale": st.scale_ms, "split": st.split_ms, "gemm": st.gemm_ms, "crt": st.crt_ms},
            "cublas_zgemm_tflops": zref, "vs_cublas_zgemm": flops / (ms * 1e-3) / 1e12 / zref}


# ------------------------------------------------------------------ the adaptive-s stream
def step_specs(a, rank):
    """the stream of this rank cut into steps: a list of (n, phi, seed) lists"""
    b = batch_size(a)
    specs = stream_specs(a.seed + 7919 * rank, min(a.problems, b * a.steps))
    return [specs[i:i + b] for i in range(0, len(specs), b)]


def over_ranks(dist, torch, world, dev, ms, flops):
    """(max over ranks of the timed region, sum over ranks of the work); identity on one rank"""
    if world <= 1:
        return ms, flops
    x = torch.tensor([ms, flops], dtype=torch.float64, device=dev)
    mx = x.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(x, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(x[1])


def problem_analytic_s(oz, batch):
    """per-problem analytic s: the largest tile analytic s of each problem"""
    out = []
    for p in batch:
        _, sa = oz.tile_features([as_args(p)], TARGET_BITS)
        out.append(int(sa.max()))
    return out


def dd_refs(oz, torch, dev, batch):
    """the double-double product hi + lo and |A||B| of every problem of the batch (untimed)"""
    refs = []
    for p in batch:
        n = p["n"]
        hi = torch.empty(n * n, dtype=torch.float64, device=dev)
        lo, ab = torch.empty_like(hi), torch.empty_like(hi)
        oz.dd_reference(n, n, n, p["A"], n, p["B"], n, hi, lo, ab)
        refs.append((hi, lo, ab))
    return refs


def check(oz, batch, refs, acc):
    """measures every output of the batch against its double-double product and adds to acc:
    problems, problems over the bound, largest ratio, largest ulp error, correctly rounded entries"""
    for p, (hi, lo, ab) in zip(batch, refs):
        n = p["n"]
        r = oz.error_ratio(n, n, n, p["C"], n, hi, lo, ab, TARGET_BITS)
        u, c = oz.accuracy(n, n, p["C"], n, hi, lo)
        acc["problems"] += 1
        acc["over_bound"] += int(r > 1.0)
        acc["max_ratio"] = max(acc["max_ratio"], r)
        acc["ulp_max"] = max(acc["ulp_max"], u)
        acc["cr_entries"] += c
        acc["entries"] += n * n


def e2e_leg(oz, torch, dev, stream, b0, steps):
    """end to end through the public API: every step copies its A and B from pinned host memory,
    makes the batched adaptive call and copies every C back. The batch lives in one pinned host
    arena per direction (inputs: every A, then every B; outputs: every C), so each direction is a
    few large copies. Two sets of device arenas let step i + 1's inputs travel (one copy stream per
    direction) while step i computes and step i - 1's results come back; each step still moves all
    of its own bytes."""
    sizes = [p["n"] ** 2 for p in b0]
    slots = [(sz + 31) // 32 * 32 for sz in sizes]  # every matrix 256-byte aligned, as allocations are
    tot = sum(slots)

    def views(buf, base):
        out, o = [], base
        for sz, sl in zip(sizes, slots):
            out.append(buf[o:o + sz])
            o += sl
        return out

    h_in = torch.empty(2 * tot, dtype=torch.float64, pin_memory=True)
    h_out = torch.empty(tot, dtype=torch.float64, pin_memory=True)
    for p, x, y in zip(b0, views(h_in, 0), views(h_in, tot)):
        x.copy_(p["A"])
        y.copy_(p["B"])
    sets = []
    for _ in range(2):
        d_in = torch.empty(2 * tot, dtype=torch.float64, device=dev)
        d_out = torch.zeros(tot, dtype=torch.float64, device=dev)
        sets.append((d_in, d_out, [dict(p, A=x, B=y, C=z) for p, x, y, z in
                                   zip(b0, views(d_in, 0), views(d_in, tot), views(d_out, 0))]))
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event()  # noqa: E731
    pieces = 8  # copies per direction and step: the first ones start moving while the rest queue

    def chunked(dst, src):
        c = (dst.numel() + pieces - 1) // pieces
        for j in range(0, dst.numel(), c):
            dst[j:j + c].copy_(src[j:j + c], non_blocking=True)

    def run(nsteps):
        ready, done, back = [ev(), ev()], [None, None], [None, None]
        start = ev()
        start.record(stream)

        def upload(i):
            h2d.wait_event(start)
            if done[i % 2] is not None:  # the compute that last read this set has finished
                h2d.wait_event(done[i % 2])
            with torch.cuda.stream(h2d):
                chunked(sets[i % 2][0], h_in)
            ready[i % 2].record(h2d)

        upload(0)
        for i in range(nsteps):
            if i + 1 < nsteps:
                upload(i + 1)
            _, d_out, probs = sets[i % 2]
            stream.wait_event(ready[i % 2])
            if back[i % 2] is not None:  # step i - 2's results have left this set's C
                stream.wait_event(back[i % 2])
            oz.gemm_adaptive([as_args(p) for p in probs], TARGET_BITS, oz.ADAPTIVE_MLP)
            done[i % 2] = ev()
            done[i % 2].record(stream)
            d2h.wait_event(done[i % 2])
            with torch.cuda.stream(d2h):
                chunked(h_out, d_out)
            back[i % 2] = ev()
            back[i % 2].record(d2h)
        for b in back:
            if b is not None:
                stream.wait_event(b)

    oz.gemm_adaptive([as_args(p) for p in b0], TARGET_BITS, oz.ADAPTIVE_MLP)  # device-resident, to compare
    run(2)
    with Timer(torch, stream) as t:
        run(steps)
    torch.cuda.synchronize()
    same = sum(int(torch.equal(p["C"].cpu().view(torch.int64), c.view(torch.int64)))
               for p, c in zip(b0, views(h_out, 0)))
    out = {"ms_per_step": t.ms / steps, "flops_per_step": flops_of(b0), "h2d": 16 * tot, "d2h": 8 * tot,
           "same": f"{same} of {len(b0)}"}
    del h_in, h_out, sets
    return out


def probe_study(a, oz, torch, dev):
    """What the probes catch: the MLP mode at lowered decision thresholds (more tiles below their
    arbiter's s) over the first batches of the stream, with no probe, the column probe, the Freivalds
    probe and both; per setting the problems over the bound after the reruns, the probed and rerun
    tiles, and the step time. Prints one JSON line."""
    model = oz.load_model()
    if a.probe_kind >= 0:
        oz.set_probe_kind(a.probe_kind)
    steps = step_specs(a, 0)
    rows = []
    for part in steps:
        batch = [make_problem(torch, dev, n, phi, sd) for n, phi, sd in part]
        refs = dd_refs(oz, torch, dev, batch)
        for thr in (0.999, 0.99, 0.95, 0.9):
            for kind, name in ((3, "none"), (0, "columns"), (1, "freivalds"), (2, "both")):
                oz.set_adaptive_options(512, thr)
                oz.set_probe_kind(kind)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                st = oz.gemm_adaptive([as_args(p) for p in batch], TARGET_BITS, oz.ADAPTIVE_MLP)
                torch.cuda.synchronize()
                ms = (time.perf_counter() - t0) * 1e3
                acc = {"problems": 0, "over_bound": 0, "max_ratio": 0.0, "ulp_max": 0.0, "cr_entries": 0,
                       "entries": 0}
                check(oz, batch, refs, acc)
                rows.append({"threshold": thr, "probe": name, "problems": acc["problems"],
                             "over_bound": acc["over_bound"], "max_ratio": acc["max_ratio"],
                             "probed": st["probed"], "rerun": st["rerun"], "ms": ms})
        del batch, refs
        torch.cuda.empty_cache()
    oz.set_probe_kind(0)
    oz.set_adaptive_options(512, model.get("threshold", 0.999))
    merged = {}
    for r in rows:
        key = (r["threshold"], r["probe"])
        m = merged.setdefault(key, {"threshold": r["threshold"], "probe": r["probe"], "problems": 0,
                                    "over_bound": 0, "max_ratio": 0.0, "probed": 0, "rerun": 0, "ms": 0.0})
        for f in ("problems", "over_bound", "probed", "rerun", "ms"):
            m[f] += r[f]
        m["max_ratio"] = max(m["max_ratio"], r["max_ratio"])
    print(json.dumps({"probe_study": list(merged.values()), "config": workload(a)}), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference_arm(a)
    import torch
    import torch.distributed as dist
    import oz2
    oz2.set_split_kernel(a.split_kernel)
    oz2.set_crt_kernel(a.crt_kernel)
    oz2.set_scale_fusion(a.scale_fusion)
    oz2.set_crt_fusion(a.crt_fusion)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    if a.dgemm_only:
        out = dgemm_leg(a, oz2, torch, dev, stream, rank)
        if rank == 0:
            print(json.dumps({"dgemm_only": out}), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    oz = oz2.Ozaki2(stream)
    oz.set_workspace_limit(WORKSPACE)
    if a.probe_study:
        probe_study(a, oz, torch, dev)
        oz.close()
        return
    model = oz.load_model()
    ref_rule = oz2.Ozaki2.moduli_for_bits
    steps = step_specs(a, rank)
    ctx = {}  # per-batch data the forms read (per-problem analytic s)

    def args_of(batch):
        return [as_args(p) for p in batch]

    # forms of the stream, each one call (or one call per problem) over a batch
    def adaptive(b):
        return oz.gemm_adaptive(args_of(b), TARGET_BITS, oz.ADAPTIVE_MLP)

    def certified_tiles(b):
        return oz.gemm_adaptive(args_of(b), TARGET_BITS, oz.ADAPTIVE_CERTIFIED_TILE)

    def certified_problem(b):
        return oz.gemm_adaptive(args_of(b), TARGET_BITS, oz.ADAPTIVE_CERTIFIED_PROBLEM)

    def analytic_batched(b):
        return oz.gemm_adaptive(args_of(b), TARGET_BITS, oz.ADAPTIVE_ANALYTIC_PROBLEM)

    def analytic_plain(b):
        for p, sv in zip(b, ctx["s_an"]):
            if sv > oz2.K_MAX_MODULI:  # no moduli set reaches the target: native FP64 (cuBLAS)
                n = p["n"]
                torch.mm(p["B"].view(n, n), p["A"].view(n, n), out=p["C"].view(n, n))
            else:
                oz.gemm(*as_args(p, sv))

    def native_fp64(b):  # cuBLAS DGEMM for every problem: DGEMM-level error by construction
        for p in b:
            n = p["n"]
            torch.mm(p["B"].view(n, n), p["A"].view(n, n), out=p["C"].view(n, n))

    def s24_grouped(b):
        oz.gemm_grouped([as_args(p, 24) for p in b])

    def refrule_grouped(b):
        oz.gemm_grouped([as_args(p, max(2, ref_rule(p["n"], TARGET_BITS))) for p in b])

    HEAD = "adaptive_mlp_batched"
    forms = {HEAD: adaptive, "adaptive_certified_batched": certified_tiles,
             "certified_per_problem_batched": certified_problem, "analytic_per_problem_batched": analytic_batched,
             "analytic_per_problem_plain_calls": analytic_plain, "native_fp64_cublas": native_fp64,
             "s24_grouped": s24_grouped, "reference_rule_grouped": refrule_grouped}
    if a.forms == "headline":
        forms = {HEAD: adaptive}
    checks = {f: {"problems": 0, "over_bound": 0, "max_ratio": 0.0, "ulp_max": 0.0, "cr_entries": 0, "entries": 0}
              for f in forms}
    ms_sum = {f: 0.0 for f in forms}
    flops_sum = 0.0
    adaptive_stats, st_sum, macs, launches = {}, [0.0] * 6, 0, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_step(fn, batch):
        """one step bracketed by a barrier and a device synchronisation on both sides, timed with
        CUDA events on the launching stream; the slowest rank's time"""
        if world > 1:
            dist.barrier()
        with NoGC():
            torch.cuda.synchronize()
            e0.record(stream)
            ret = fn(batch)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            x = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            ms = float(x[0])
        return ms, ret

    # warm-up: every form on the first batch (also sizes the workspaces)
    batch = [make_problem(torch, dev, n, phi, sd) for n, phi, sd in steps[0]]
    ctx["s_an"] = problem_analytic_s(oz, batch)
    for _ in range(a.warmup):
        for fn in forms.values():
            fn(batch)
    torch.cuda.synchronize()
    oz.check_device_error()

    # timed steps: each batch generated (untimed), then every form timed on it and checked
    by_form = {}
    gbytes = [0, 0, 0]
    with ClockSampler(local) as clk:
        for i, part in enumerate(steps):
            if i > 0:
                del batch
                torch.cuda.empty_cache()
                batch = [make_problem(torch, dev, n, phi, sd) for n, phi, sd in part]
                ctx["s_an"] = problem_analytic_s(oz, batch)
            refs = dd_refs(oz, torch, dev, batch)
            flops_sum += flops_of(batch)
            for name, fn in forms.items():
                l0 = oz.kernel_launches() if name == HEAD else 0
                if name == HEAD:
                    torch.cuda.nvtx.range_push("headline")
                ms, ret = timed_step(fn, batch)
                if name == HEAD:
                    torch.cuda.nvtx.range_pop()
                    launches += oz.kernel_launches() - l0
                    for key, v in ret.items():
                        adaptive_stats[key] = adaptive_stats.get(key, 0) + v
                ms_sum[name] += ms
                check(oz, batch, refs, checks[name])
            # stage times and the GEMM against the int8 roofline: a profiling pass of the headline
            # form on the same batch (untimed)
            oz.set_profiling(True)
            st = adaptive(batch)
            macs += st["int8_macs"]
            tt, at = oz.stage_times(), oz.adaptive_stage_times()
            for j, v in enumerate((tt.scale_ms, tt.split_ms, tt.gemm_ms, tt.crt_ms, at["probe_ms"], at["native_ms"])):
                st_sum[j] += v
            oz.set_profiling(False)
            gb = oz.adaptive_gemm_bytes()
            gbytes = [gbytes[0] + gb["plane_bytes"], gbytes[1] + gb["residue_bytes"], gbytes[2] + gb["batches"]]
            if i == 0:  # the stage times of every adaptive-call form on the first batch (untimed)
                for name, fn in forms.items():
                    if fn not in (adaptive, certified_tiles, certified_problem, analytic_batched):
                        continue
                    oz.set_profiling(True)
                    fn(batch)
                    tt, at = oz.stage_times(), oz.adaptive_stage_times()
                    oz.set_profiling(False)
                    by_form[name] = {"scale_stats": tt.scale_ms, "split": tt.split_ms, "gemm": tt.gemm_ms,
                                     "crt": tt.crt_ms, "probe": at["probe_ms"], "native_fp64": at["native_ms"]}
            del refs
            if rank == 0:
                print(f"step {i + 1}/{len(steps)}: {len(batch)} problems, headline {ms_sum[HEAD]:.1f} ms so far, "
                      f"device memory peak {torch.cuda.max_memory_allocated() / 2 ** 30:.1f} GiB", file=sys.stderr,
                      flush=True)
    oz.check_device_error()
    nsteps = len(steps)
    _, flops_all = over_ranks(dist, torch, world, dev, 0.0, flops_sum)
    value = flops_all / (ms_sum[HEAD] * 1e-3) / 1e12
    peak, note = int8_peak()
    achieved = 2.0 * macs / (st_sum[2] * 1e-3) / 1e12

    def summary_of(c):
        return {"problems": c["problems"], "over_bound": c["over_bound"], "max_ratio": c["max_ratio"],
                "ulp_max": c["ulp_max"], "cr_frac": c["cr_entries"] / max(c["entries"], 1)}

    fixed = {name: {"tflops": flops_all / (ms_sum[name] * 1e-3) / 1e12, "ms_per_step": ms_sum[name] / nsteps,
                    "adaptive_speedup": ms_sum[name] / ms_sum[HEAD]} for name in forms if name != HEAD}
    tiles = max(adaptive_stats.get("tiles", 0), 1)
    emulated = max(tiles + adaptive_stats.get("rerun", 0) - adaptive_stats.get("native_tiles", 0), 1)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": nsteps, "warmup": a.warmup,
            "ms_per_step": ms_sum[HEAD] / nsteps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (int8 residues, int32 accumulate)", "data": "synthetic",
            "config": dict(workload(a), model_threshold=model.get("threshold"), workspace_limit_gib=WORKSPACE >> 30),
            "clocks": clk.summary(), "gpu_launches": launches,
            "stage_ms_per_step": {"scale_stats_mlp": st_sum[0] / nsteps, "split": st_sum[1] / nsteps,
                                  "gemm": st_sum[2] / nsteps, "crt": st_sum[3] / nsteps,
                                  "probe": st_sum[4] / nsteps, "native_fp64": st_sum[5] / nsteps},
            "roofline": {"bound": "tensor", "kernel": "gemm_i8_modm_kernel", "achieved": achieved, "peak": peak,
                         "unit": "TOPS (int8)", "frac": achieved / peak, "peak_note": note,
                         "algorithmic": "2 s m_t n_t k int8 ops per tile (reruns included), summed over the steps",
                         "algorithmic_bytes_per_launch": (gbytes[0] + gbytes[1]) / max(gbytes[2], 1),
                         "launches": gbytes[2],
                         "traffic": GEMM_TRAFFIC_RATIO * (gbytes[0] + gbytes[1]) / max(gbytes[2], 1),
                         "traffic_note": "DRAM bytes per launch: the measured DRAM/algorithmic ratio of an ncu "
                                         "capture of a small case of this stream times this run's algorithmic "
                                         "bytes per launch (planes read once, residues written)"},
            "stage_ms_first_batch_by_form": by_form,
            "fixed_s": fixed,
            "error_check": {"bound": "|C - AB| <= k 2^-53 (|A||B|)_ij against a double-double product, per entry; "
                                     "ulp_max in units of the spacing above |AB|, cr_frac = entries equal to RN(AB)",
                            **{f: summary_of(c) for f, c in checks.items()}},
            "adaptive_tiles": {"tiles": adaptive_stats.get("tiles"),
                               "native_tiles": adaptive_stats.get("native_tiles"),
                               "mean_s_emulated": adaptive_stats.get("sum_s", 0) / emulated,
                               "mean_analytic_s": adaptive_stats.get("analytic_sum_s", 0) / tiles,
                               "analytic_note": "33 counts a tile the analytic rule sends to native FP64",
                               "probed": adaptive_stats.get("probed"), "rerun": adaptive_stats.get("rerun")}}
    del batch
    torch.cuda.empty_cache()

    # end to end with host buffers, on the first E2E_BATCH problems of the stream
    b0 = [make_problem(torch, dev, n, phi, sd) for n, phi, sd in steps[0][:E2E_BATCH]]
    e2e_steps = max(2, a.steps)  # the pipeline's fill and drain amortised over the steps
    e = e2e_leg(oz, torch, dev, stream, b0, e2e_steps)
    e2e_ms, e2e_flops = over_ranks(dist, torch, world, dev, e["ms_per_step"], e["flops_per_step"])
    line["e2e"] = {"value": e2e_flops / (e2e_ms * 1e-3) / 1e12, "unit": UNIT,
                   "h2d_bytes_per_step": e["h2d"], "d2h_bytes_per_step": e["d2h"], "ms_per_step": e2e_ms,
                   "steps": e2e_steps, "outputs_equal_device_call": e["same"],
                   "note": f"the first {len(b0)} problems of the stream every step (one adaptive call), from one "
                           "pinned host arena per direction (8 copies each); step i + 1's inputs copy in while step "
                           "i computes and step i - 1's results copy out (two device arena sets, one copy stream "
                           "per direction)"}
    del b0
    oz.check_device_error()
    oz.close()
    torch.cuda.empty_cache()

    extras = {}
    if not a.no_extras:
        extras["dgemm_8192"] = dgemm_leg(a, oz2, torch, dev, stream, rank)
        extras["zgemm_4096"] = zgemm_leg(oz2, torch, dev, stream, rank)
        extras["grouped_c4"] = grouped_leg(oz2, torch, dev, stream)
        if world > 1:
            extras["dgemm_8192_sharded"] = sharded_leg(a, oz2, torch, dev, stream, dist, world, rank)
        if world == 1:  # the host-core baselines are quoted at one GPU only
            line["cpu_baseline"] = cpu_sample(a)
            line["cpu_baseline_dgemm"] = cpu_dgemm_sample(a)
    line["extras"] = extras
    # last, where a truncated log keeps it: the headline's accuracy and its speed-up over each form
    hc = checks[HEAD]
    line["summary"] = {"problems_timed": hc["problems"], "over_bound": hc["over_bound"],
                       "max_ratio": hc["max_ratio"], "ulp_max": hc["ulp_max"],
                       "cr_frac": hc["cr_entries"] / max(hc["entries"], 1),
                       "speedup_over": {f: round(v["adaptive_speedup"], 3) for f, v in fixed.items()},
                       "forms_over_bound": {f: c["over_bound"] for f, c in checks.items()},
                       "roofline_frac": round(achieved / peak, 3), "e2e": line["e2e"]["value"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
