"""bench.py's reference arm on the host: one JSON line with the contract's keys from rank 0 (the
reference's own CPU path, or the C oracle where the reference was not built), nothing and exit
status 0 from the other ranks. CPU only."""
import json
import os
import subprocess
import sys

from common import ROOT


def run_arm(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    return [line for line in r.stdout.splitlines() if line.startswith("{")]


def test_reference_arm_prints_the_contract_line():
    lines = run_arm({"RANK": "0", "WORLD_SIZE": "1"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["higher_is_better"] is True and d["steps"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("adaptive-s stream")


def test_reference_arm_other_ranks_print_nothing():
    assert run_arm({"RANK": "1", "WORLD_SIZE": "2"}) == []


def _stream(monkeypatch, s_value, status=0):
    import importlib
    import types
    sys.path.insert(0, ROOT)
    bench = importlib.import_module("bench")
    a = types.SimpleNamespace(seed=2025, problems=3, steps=1, batch=0)
    cs = bench.CpuStream(a)
    cs.specs = [(64, 1.0, 11), (96, 2.0, 12), (80, 0.5, 13)]  # small problems of the stream's kind
    monkeypatch.setattr(cs.ao, "problem_analytic_s", lambda *args, **kw: s_value)
    if status:
        monkeypatch.setattr(cs.lib, "dgemm", lambda *args, **kw: (status, None))
    return cs


def test_cpu_stream_runs_problems_beyond_24_moduli_as_host_dgemm(monkeypatch):
    cs = _stream(monkeypatch, 25)
    flops, secs = cs.step(60.0)
    assert cs.native == 3 and cs.emulated == 0
    assert flops == 2.0 * (64 ** 3 + 96 ** 3 + 80 ** 3) and secs > 0


def test_cpu_stream_runs_the_reference_at_the_analytic_s(monkeypatch):
    cs = _stream(monkeypatch, 20)
    flops, secs = cs.step(60.0)
    assert cs.emulated == 3 and cs.native == 0 and secs > 0


def test_cpu_stream_fails_loudly_on_a_failed_call(monkeypatch):
    import pytest
    cs = _stream(monkeypatch, 20, status=1)
    with pytest.raises(RuntimeError):
        cs.step(60.0)
