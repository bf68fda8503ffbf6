"""The reference arm's JSON line (``bench.py --impl reference``): one line on
rank 0 with the keys, metric, unit and config of the device arm, an ``e2e``
object with no host<->device bytes, a ``cpu_baseline`` that describes the run,
and step counts that are the ones actually run (each step is one complete
matvec; the arm stops early at its time budget).  The oracle matvec itself is
replaced by a fixed-duration stand-in here (a real one takes ~45 s of host
time); the device arm's config carries no measured results."""
import argparse
import contextlib
import io
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _run(monkeypatch, rank, steps=3, warmup=3, budget=60.0, dt=0.01):
    calls = {"full": [], "short": 0}

    def fake_fn():
        def f(i, cap=None):
            if cap is None:
                calls["full"].append(i)
                time.sleep(dt)
            else:
                calls["short"] += 1
        return f

    monkeypatch.setattr(bench, "oracle_matvec_fn", fake_fn)
    args = argparse.Namespace(gpus=2, steps=steps, warmup=warmup)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, rank, budget_s=budget)
    return buf.getvalue(), calls


def test_reference_line_contract(monkeypatch):
    out, calls = _run(monkeypatch, 0)
    lines = [ln for ln in out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["config"] == bench.workload_config()
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["value"] == d["cpu_baseline"]["value"] == d["e2e"]["value"]
    assert d["e2e"]["unit"] == bench.UNIT
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (2, 3, 3)
    assert calls["full"] == [0, 1, 2] and calls["short"] == 3       # one complete matvec per step
    assert d["step"]["matvecs"] == 1
    # one step = one matvec: value * ms_per_step = 1000, and steps x ms_per_step is the timed work
    assert abs(d["value"] * d["ms_per_step"] - 1e3) < 1e-6
    assert 0.009 * 3 < d["steps"] * d["ms_per_step"] / 1e3 < 1.0


def test_reference_arm_stops_at_its_budget(monkeypatch):
    """Requested 20 steps of 10 ms with a 25 ms budget: the arm stops after the
    step that would overrun and reports the 2 steps it ran."""
    out, calls = _run(monkeypatch, 0, steps=20, budget=0.025)
    d = json.loads(out)
    assert d["steps"] == 2 == len(calls["full"]) and d["step"]["requested_steps"] == 20


def test_reference_arm_other_ranks_do_nothing(monkeypatch):
    out, calls = _run(monkeypatch, 1)
    assert out == "" and calls == {"full": [], "short": 0}


def test_device_config_carries_no_results():
    cfg = bench.workload_config()
    for k in ("adaptive_info", "secondary", "phase_ms", "tangents_per_step"):
        assert k not in cfg
    assert json.loads(json.dumps(cfg)) == cfg


def test_tangent_kernel_bytes_match_the_box_layout():
    """n=128 FP64 (K=43, M=85), 64 tangents: 39,976,960 B for the row pass and
    54,540,512 B for the column pass; the HBM model's tangent RHS is 2 x 1,056,768 B."""
    row, col = bench.tangent_kernel_bytes(43, 85, 64)
    assert row == 64 * 7 * 43 * 128 * 16 + 128 * 4 * 128 * 8 == 39976960
    assert col == 64 * (7 * 43 * 128 * 16 + 2 * 7310 * 16) + 7310 * 16
    assert bench.tangent_rhs_model_bytes() == 2 * 1056768
