"""The bench's reference arm runs the CPU checker only: it must load none of this
repository's CUDA code and print the same ``config`` as the GPU arm."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
import bench
bench.H3_SAMPLE = dict(nrefine=0, nrhs=1)
bench.run_reference(bench.parse())
maps = open("/proc/self/maps").read()
print(json.dumps({"libqbxfmm_loaded": "libqbxfmm" in maps,
                  "config": bench.config_dict(bench.parse(), 1)}))
"""


def test_reference_arm_loads_no_cuda_library_and_matches_config():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    res = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    lines = [json.loads(ln) for ln in res.stdout.splitlines() if ln.startswith("{")]
    ref, check = lines[0], lines[1]
    assert ref["impl"] == "reference" and ref["value"] > 0
    assert ref["cpu_baseline"]["kind"] == "port"
    assert not check["libqbxfmm_loaded"]
    assert ref["config"] == check["config"]
