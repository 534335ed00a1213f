"""bench.py's reference arm on the CPU: one JSON line with the keys the
benchmark contract names, on the small 2D workload (256x256 blobs), and the
rank helpers without a process group."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

REQUIRED = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
            "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"]


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "blobs2d",
                        "--steps", "3", "--warmup", "3"], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in REQUIRED:
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["steps"] == 3 and d["warmup"] >= 3
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["voxels_per_step"] == 256 * 256


def test_rank_helpers_single_process():
    sys.path.insert(0, ROOT)
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(2.5, 1) == 2.5
