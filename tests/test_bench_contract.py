"""The bench's reference arm (the C oracle port on the host cores) runs without a
GPU, so its JSON line is checked here against the bench contract: one line,
the same metric and unit as the engine arm, a bounded CPU sample described in
`cpu_baseline`, a host-only `e2e`, and nothing printed by ranks other than 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _run(args, env=None):
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                         timeout=600, env=env, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    return res.stdout


@pytest.mark.parametrize("workload", ["config2", "config1"])
def test_reference_arm_line_follows_the_contract(workload):
    out = _run(["--impl", "reference", "--workload", workload, "--steps", "3", "--warmup", "3"])
    lines = [l for l in out.splitlines() if l.strip()]
    assert len(lines) == 1, out
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"] == bench.workload_config(workload)   # the engine arm prints the same object
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["unit"] == "steps/s" and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == "steps/s"
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_prints_nothing_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert _run(["--impl", "reference", "--steps", "3", "--warmup", "3"], env=env).strip() == ""


def test_algorithmic_work_per_step():
    """The roofline numerators: bytes 2 (N_src + N_tgt) n 4 per step (each side's
    block read and written once), and the multiply-adds of d, D d^T and the
    projection, at the two synthetic sizes the bench reports."""
    c2 = bench.algorithmic(bench.shape_of("config2"))
    assert c2["step_bytes"] == 2 * (1847560 + 2116296) * 16 * 4            # 0.507 GB
    assert abs(c2["step_bytes"] / 1e9 - 0.507) < 0.001
    assert c2["macs"] == 2 * 75582 * 11 * 28 * 20 * 16 + 1847560 * 16 * 16
    c5 = bench.algorithmic(bench.shape_of("config5"))
    assert c5["step_bytes"] == 2 * (43266496 + 45762640) * 32 * 4          # 22.79 GB
    assert abs(c5["step_bytes"] / 1e9 - 22.79) < 0.01
    assert c5["macs"] == 2 * 1144066 * 13 * 40 * 32 * 32 + 43266496 * 32 * 32


def test_peak_file_falls_back_when_unreadable(tmp_path, monkeypatch):
    """A missing or malformed peaks file gives the stated fallback, never an error."""
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text("{not json")
    assert bench.measured_peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6457.4, "bf16_tflops": 1590}))
    assert bench.measured_peaks() == (6457.4, "measured")
