"""The reference arm of bench.py (the reference's own CPU detector from
oracle/_ref on the host cores) prints one JSON line with the bench contract's
keys and the GPU arm's own `config`, and loads nothing of the GPU library; it
needs no GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# run the arm in-process, then report whether the GPU library was mapped
RUNNER = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3", "--batch", "2"]
runpy.run_path("bench.py", run_name="__main__")
print("MAPPED_GPU_LIBRARY", "libapriltag_b200" in open("/proc/self/maps").read())
"""


def test_reference_arm_json_line():
    p = subprocess.run([sys.executable, "-c", RUNNER], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    assert "MAPPED_GPU_LIBRARY False" in p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # oracle/_ref not built in this checkout
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "frames/s" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    sys.path.insert(0, ROOT)
    import bench

    assert d["config"] == bench.workload_config(2, 1)
    assert d["metric"] == bench.METRIC
