"""The reference arm's JSON line (``bench.py --impl reference``): one line on
rank 0 with the keys, metric, unit and config of the device arm, an ``e2e``
object with no host<->device bytes, and a ``cpu_baseline`` that describes the
run.  The timed CPU sample itself is replaced by a fixed result here (it takes
seconds of host time); its own sizing is covered by the bench run."""
import argparse
import contextlib
import io
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _run(monkeypatch, rank):
    fake = {"value": 0.02, "unit": bench.UNIT, "cores": 4, "kind": "port", "sample": "fixed"}
    seen = {}

    def cpu_baseline(target_s=12.0, attempts_full=None):
        seen["attempts_full"] = attempts_full
        return dict(fake)

    monkeypatch.setattr(bench, "cpu_baseline", cpu_baseline)
    args = argparse.Namespace(gpus=2, steps=3, warmup=3)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, rank)
    return buf.getvalue(), seen


def test_reference_line_contract(monkeypatch):
    out, seen = _run(monkeypatch, 0)
    lines = [ln for ln in out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["config"] == bench.workload_config()
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["value"] == d["cpu_baseline"]["value"] == d["e2e"]["value"] == 0.02
    assert d["e2e"]["unit"] == bench.UNIT
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert abs(d["ms_per_step"] - bench.BATCH / 0.02 * 1e3) < 1e-6    # one step = BATCH matvecs
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (2, 3, 3)
    assert seen["attempts_full"] > 0                                   # scaled to a full matvec


def test_reference_arm_other_ranks_do_nothing(monkeypatch):
    out, seen = _run(monkeypatch, 1)
    assert out == "" and seen == {}
