"""bench.py's reference arm runs on the host cores without a GPU: the GPU arm's step
(pairs per step, distinct pairs), every requested step, one JSON line with the fields the
comparison reads.  A small frame size keeps it to seconds."""
import json
import os
import subprocess
import sys

from conftest import REPO


def test_reference_arm_json_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "3",
                          "--warmup", "1", "--size", "128", "--pairs", "4"],
                         capture_output=True, text=True, timeout=600, env=env, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 3 and d["unit"] == "pairs/s" and d["value"] > 0
    assert d["higher_is_better"] is True
    assert d["config"]["pairs_per_step_per_gpu"] == 4 and d["config"]["unique_pairs"] == 4
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
