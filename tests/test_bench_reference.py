"""The bench's reference arm (`bench.py --impl reference`): the reference's own
step loop (oracle/_ref/slab_ref, built from the reference's sources) timed on
the host cores, printed as one JSON line with the fields of the product arm's
line. The W warm-up steps are untimed: the run puts an output frame after
them and times the steps between that frame and the last one. Runs on the
small 35-degree slope workload so it takes about a second."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(O.REF_BIN), reason="reference binary not built")
def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c1", "--steps", "3",
                        "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == d["metric"] and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] >= 3  # at least one frame of 3 steps after the warm-up
    assert d["warmup"] == 3
    assert d["config"]["workload"] == "slope35_arc_401x101_dx5" and d["config"]["particles"] == 1600
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["repo_libraries_loaded"] == []  # the reference arm runs none of this repository's native code
