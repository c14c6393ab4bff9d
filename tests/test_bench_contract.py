"""The JSON line of `bench.py --impl reference` (the reference solver timed on
the host cores) on a tiny case, and the workload description of both arms.
Host only: the reference arm runs no GPU code."""
import json
import os
import subprocess
import sys

import pytest
from conftest import REPO

sys.path.insert(0, REPO)
import bench  # noqa: E402

KEYS = {"metric": str, "value": float, "unit": str, "n_gpus": int, "steps": int, "warmup": int,
        "ms_per_step": float, "higher_is_better": bool, "scaling": str, "dtype": str, "data": str,
        "config": dict, "impl": str, "cpu_baseline": dict, "e2e": dict}


@pytest.mark.skipif(not os.path.exists(bench.REFDRIVER), reason="reference driver not built")
def test_reference_arm_line(tmp_path):
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--n", "6", "--blocks", "2"], cwd=tmp_path, capture_output=True,
                         text=True, timeout=300, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k, t in KEYS.items():
        assert isinstance(line[k], t), k
    assert line["impl"] == "reference" and line["vs_baseline"] is None and line["value"] > 0
    assert line["metric"] == "cell-iters/s" and line["higher_is_better"] is True
    assert line["config"]["cells"] == 6 * 6 ** 3 and line["config"]["blocks"] == 2
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "less than the 126 MB L2" in line["config"]["l2"]


def test_workload_l2_statement():
    assert "more than the 126 MB L2" in bench.workload_config(80, 16, "fp32")["l2"]
    assert "more than the 126 MB L2" in bench.workload_config(48, 16, "fp32")["l2"]
    assert "less than the 126 MB L2" in bench.workload_config(8, 2, "fp64")["l2"]
