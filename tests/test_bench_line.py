"""The JSON line bench.py prints, checked without a GPU: bench.main runs with
the measuring functions replaced by synthetic results, and the line must
carry the keys, units and objects the benchmark contract names (the
roofline with its achieved / peak / frac / traffic, the CPU baseline, the
end-to-end figure with the bytes copied per step, clocks, launches), the
mixed form's errors after the 100 steps, and a sidecar that keeps the
solve's per-phase and per-level breakdown the line leaves out."""

import importlib.util
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_line", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _errors(phi, rho):
    return {"comparable": True, "steps": 100, "phi_rel_l2": phi, "rho_rel_l1": rho, "lz_total_rel": 1e-12,
            "growth": [{"comparable": True, "steps": 1, "phi_rel_l2": phi / 2, "rho_rel_l1": rho / 2}]}


def _head():
    per_level = [1.0, 2.0, 3.0]
    return {
        "value": 3.4e6, "ms_per_step": 136.0, "ms_steps": [130.0, 142.0], "bricks": 315,
        "leaf_cells_per_step": 469692.0,
        "e2e": {"value": 3.3e6, "unit": "cell-updates/s", "h2d_bytes_per_step": 188326944,
                "d2h_bytes_per_step": 188781840, "ms_per_step": 142.5, "ms_steps": [140.0, 145.0]},
        "autotune": {"layout": 1, "blocks_per_sm": 1, "threads": 864, "blocks": 148, "trials_ms": [1.0, None]},
        "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 5},
        "gpu_launches": 926,
        "persistent": {"bytes_per_launch": 1.0e10, "ms_per_launch": 40.0,
                       "phase_ms_per_step": {"relax": 100.0}, "phases_per_step": {"relax": 3000.0},
                       "barrier_ms_per_step": {"relax": 2.0}, "level_sum_ms_per_step": 10.0,
                       "bricks_by_level": [1, 8, 32], "relax_passes_per_step_by_level": per_level,
                       "relax_split_per_step": {"pass_ms": 60.0}, "relax_ms_per_step_by_level": per_level},
    }


def _ztwd():
    form = {"value": 1.0e6, "ms_per_step": 400.0, "gpu_launches_total": 3046025}
    return {"fp64": form, "fp64_persistent": dict(form, ms_per_step=186.0), "mixed": dict(form, ms_per_step=134.0),
            "mixed_flux32": dict(form, ms_per_step=133.0),
            "errors_mixed_vs_fp64": _errors(4.9e-10, 7.5e-11), "errors_mixed_flux32_vs_fp64": _errors(8.6e-9, 6.6e-8),
            "cpu_baseline": {"value": 1.85e4, "unit": "cell-updates/s", "cores": 16, "kind": "reference",
                             "sample": "synthetic"}}


def test_bench_line_keeps_the_contract(tmp_path, monkeypatch, capsys):
    bench = _bench()
    import torch
    monkeypatch.setattr(torch.cuda, "set_device", lambda *a, **k: None)
    monkeypatch.setattr(bench, "load_amr", lambda: (None, type("Ini", (), {"BINARY": {"q": 0.7}})))
    monkeypatch.setattr(bench, "run_ztwd_headline", lambda *a, **k: _head())
    monkeypatch.setattr(bench, "run_ztwd", lambda *a, **k: _ztwd())
    side = tmp_path / "side.json"
    monkeypatch.setattr(sys, "argv", ["bench.py", "--json-out", str(side)])
    assert bench.main() == 0
    lines = [x for x in capsys.readouterr().out.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "clocks", "gpu_launches"):
        assert k in line, k
    assert line["n_gpus"] == 1 and line["higher_is_better"] is True and line["unit"] == "cell-updates/s"
    assert "workload" in line["config"] and "l2" in line["config"]
    r = line["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert abs(r["achieved"] - 1.0e10 / 0.040 / 1e9) < 1e-9 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert "traffic" in r and "phase_ms_per_step" not in r
    e = line["e2e"]
    assert {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"} <= set(e)
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 16
    assert line["errors_vs_fp64"]["phi_rel_l2"] == 4.9e-10 and "growth" not in line["errors_vs_fp64"]
    assert line["speedup_vs_fp64_plain"] == 400.0 / 136.0
    assert line["mixed_flux32_100_steps"]["rho_rel_l1"] == 6.6e-8
    assert len(lines[0]) < 4000
    s = json.loads(side.read_text())
    assert s["roofline"]["relax_ms_per_step_by_level"] == [1.0, 2.0, 3.0]
    assert s["ztwd_binary"]["errors_mixed_vs_fp64"]["growth"]


def test_reference_arm_line(monkeypatch, capsys):
    """--impl reference: the line of the reference's own CPU build, on the
    same metric and workload, with its CPU description and an end-to-end
    figure that copies nothing; without the harness it says why in one
    line."""
    bench = _bench()
    sample = {"seconds": [25.0, 25.5], "leaf_cells": [467424, 467424], "threads": 16, "bricks": 309}
    monkeypatch.setattr(bench, "run_reference_ztwd", lambda *a, **k: sample)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    assert bench.main() == 0
    line = json.loads([x for x in capsys.readouterr().out.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert abs(line["value"] - 2 * 467424 / 50.5) < 1e-9
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 16
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["config"]["workload"] == bench.ZT_WORKLOAD % bench.ZT_NX
    monkeypatch.setattr(bench, "run_reference_ztwd", lambda *a, **k: None)
    assert bench.main() == 0
    line = json.loads([x for x in capsys.readouterr().out.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and "unavailable" in line
