"""bench.py's reference arm (CPU only): the compiled reference timed on a row
band of the 1080p workload, one JSON line with the contract's keys; ranks
other than 0 print nothing and exit 0."""
import json
import os
import subprocess
import sys

import pytest

from oracle.lenia_oracle import RefLenia

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(extra_env=None, *args):
    env = dict(os.environ, **(extra_env or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


@pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built (reference tree absent)")
def test_reference_arm_prints_one_contract_line():
    p = run_bench(None, "--steps", "2", "--warmup", "1")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [x for x in p.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Lenia Mpixel-steps/s (FFT, 3 kernels, 1080p)"
    assert d["unit"] == "Mpixel-steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"] == "fft3_1080p"
    assert (d["config"]["width"], d["config"]["height"]) == (1920, 1080)
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert "rows 0..32" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Mpixel-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = run_bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--steps", "2", "--warmup", "1")
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_traffic_comes_only_from_a_named_capture(tmp_path, monkeypatch):
    """roofline.traffic is the DRAM traffic of an ncu capture of the same
    workload, with its command as the source; absent, another workload or an
    unreadable file: null, never a constant."""
    sys.path.insert(0, ROOT)
    import bench

    f = tmp_path / "traffic.json"
    monkeypatch.setattr(bench, "TRAFFIC_FILE", str(f))
    assert bench.captured_traffic("row_growth", "fft3_1080p") == (None, None)
    f.write_text(json.dumps({"workload": "fft3_1080p", "command": "ncu ... bench.py", "note": "one launch",
                             "kernels": {"row_growth": {"dram_bytes_per_launch": 123}}}))
    t, src = bench.captured_traffic("row_growth", "fft3_1080p")
    assert t == 123 and "ncu ... bench.py" in src
    assert bench.captured_traffic("column", "fft3_1080p") == (None, None)
    assert bench.captured_traffic("row_growth", "single_256") == (None, None)
    f.write_text("{not json")
    assert bench.captured_traffic("row_growth", "fft3_1080p") == (None, None)
