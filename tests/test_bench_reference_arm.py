"""bench.py --impl reference on the host: one JSON line with the reference
arm's keys, the same workload config as the CUDA arm, a cpu_baseline that
describes the run, and an e2e entry with no host-device traffic."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libqmb_ref.so")),
                    reason="the reference's host build (oracle/_ref) is absent")
def test_reference_arm_line():
    import bench
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--cpu-seconds", "1"], check=True, capture_output=True, text=True,
                         cwd=ROOT, timeout=600).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "Hv/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["config"] == bench.batched_config(1)
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "Hv/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
