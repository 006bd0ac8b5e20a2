"""The ensemble leg of bench.py's default line (host logic, no GPU): the child
run's JSON line is summarised, and a child that fails or prints no line gives
an `error` entry instead of ending the benchmark."""

from __future__ import annotations

import importlib.util
import json
import subprocess
from pathlib import Path

BENCH = Path(__file__).resolve().parent.parent / "bench.py"


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", BENCH)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _fake_run(stdout: str, returncode: int = 0, stderr: str = ""):
    def run(cmd, **kw):
        assert "--workload" in cmd and cmd[cmd.index("--workload") + 1] == "ensemble"
        return subprocess.CompletedProcess(cmd, returncode, stdout=stdout, stderr=stderr)
    return run


def test_summary_of_child_line(monkeypatch):
    b = _bench()
    line = {"config": {"workload": "ensemble_12_domains_graph", "columns_per_step": 916631,
                       "schedule": {"streams": 1}},
            "value": 2.96e6, "ms_per_step": 309.7, "sequential_value": 2.91e6, "sequential_ms_per_step": 315.0,
            "latency_p50_ms": 7.3, "latency_p99_ms": 309.0, "sequential_latency_p50_ms": 155.0,
            "sequential_latency_p99_ms": 315.0, "fallback_columns": 251, "autotune_trials": 14,
            "clocks": {"sm_mhz": 1965.0}}
    monkeypatch.setattr(b.subprocess, "run", _fake_run("log line\n" + json.dumps(line) + "\n"))
    out = b.ensemble_leg()
    assert out["workload"] == "ensemble_12_domains_graph" and out["columns_per_step"] == 916631
    assert out["value"] == 2.96e6 and out["sequential_value"] == 2.91e6
    assert out["latency_p50_ms"] == 7.3 and out["schedule"] == {"streams": 1}
    assert "error" not in out


def test_failed_child_gives_error_entry(monkeypatch):
    b = _bench()
    monkeypatch.setattr(b.subprocess, "run", _fake_run("", returncode=1, stderr="Traceback\nRuntimeError: boom\n"))
    out = b.ensemble_leg()
    assert set(out) == {"error"} and "exited 1" in out["error"] and "boom" in out["error"]


def test_child_without_line_gives_error_entry(monkeypatch):
    b = _bench()
    monkeypatch.setattr(b.subprocess, "run", _fake_run("no json here\n"))
    assert "error" in b.ensemble_leg()


def test_timeout_gives_error_entry(monkeypatch):
    b = _bench()

    def run(cmd, **kw):
        raise subprocess.TimeoutExpired(cmd, kw.get("timeout", 0))
    monkeypatch.setattr(b.subprocess, "run", run)
    assert "exceeded" in b.ensemble_leg(timeout_s=5)["error"]
