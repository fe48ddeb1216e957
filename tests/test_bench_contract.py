"""bench.py's reference arm runs on CPU and prints one JSON line with the
keys the driver reads (the GPU arm prints the same keys plus roofline, clocks
and launch counts; it is exercised by the GPU runs).  The workload is scaled
down here (--npart) so the CPU suite stays short; the default run times the
full 256^3 box.  Both arms print the same config."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--npart", "262144"], capture_output=True, text=True, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "Mpart/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["value"] > 0
    assert "workload" in d["config"]
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    sys.path.insert(0, REPO)
    import bench
    assert d["metric"] == bench.METRIC
    assert d["config"] == bench.workload_config(bench._scaled(dict(bench.WORKLOAD), 262144), 1)
    assert d["config"]["npart"] == 262144
