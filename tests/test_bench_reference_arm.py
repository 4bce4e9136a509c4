"""bench.py --impl reference on the host: one JSON line with the reference
arm's keys, the same workload config as the CUDA arm, a cpu_baseline that
describes the run, an e2e entry with no host-device traffic, and a process
that never imports or maps the product library."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libqmb_ref.so")),
                               reason="the reference's host build (oracle/_ref) is absent")

_ARM = """
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "3", "--warmup", "1"]
sys.path.insert(0, {root!r})
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({{"product_imported": "qmbcuda_b200" in sys.modules,
                  "product_mapped": "libqmb_b200" in maps,
                  "reference_mapped": "libqmb_ref" in maps}}))
"""


@needs_ref
def test_reference_arm_line_and_isolation():
    import bench
    out = subprocess.run([sys.executable, "-c", _ARM.format(root=ROOT)], check=True, capture_output=True,
                         text=True, cwd=ROOT, timeout=600).stdout
    lines = out.strip().splitlines()
    line, probe = json.loads(lines[-2]), json.loads(lines[-1])
    # the arm runs the reference's code and nothing of the product
    assert probe == {"product_imported": False, "product_mapped": False, "reference_mapped": True}
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "Hv/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["config"] == bench.batched_config(1)
    # steps are timed sweeps over the sampled matrices, ms_per_step is one sweep
    assert line["steps"] == 3 and line["warmup"] == 1 and len(line["ms_steps"]) == 3
    assert abs(line["ms_per_step"] - np.mean(line["ms_steps"])) < 1e-2
    n_mats = 2 * 20
    assert abs(line["value"] - n_mats / (line["ms_per_step"] * 1e-3)) < 1e-6 * line["value"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "real parts" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "Hv/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@needs_ref
def test_reference_arm_inputs_equal_the_products_tables():
    """The oracle's group and term tables that the reference arm feeds to the
    reference's kernels are the ones the CUDA arm builds its batch from."""
    import oracle as O
    import qmbcuda_b200 as q
    L = 20
    perm, ch = q.translation_group(L)
    g = O.translation_group(L)
    assert np.array_equal(perm, g.perm)
    assert np.abs(ch - g.chars).max() < 1e-12
    J, D = 1.3, 0.7
    t = q.xxz_terms(q.chain_bonds(L), J, J * D)
    o = O.xxz_terms(O.chain_bonds(L), J, J * D)
    assert np.array_equal(t.n_ops, o.n_ops)
    assert np.array_equal(t.codes.ravel(), o.codes)
    assert np.array_equal(t.sites.ravel(), o.sites)
    assert np.array_equal(t.scalar, o.scalar)
