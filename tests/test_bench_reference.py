"""bench.py's reference arm on the CPU: rank 0 times the reference's own code
(the oracle built from the reference's sources) and prints one JSON line
with the contract's keys; any other rank of a multi-GPU launch exits 0
without work."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref_c

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra, *args):
    env = dict(os.environ, OMP_NUM_THREADS="2", **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)


def test_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--gpus", "2")
    assert r.returncode == 0 and r.stdout.strip() == ""


@pytest.mark.skipif(not ref_c.available(3), reason="oracle/_ref not built")
def test_rank0_prints_the_contract_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1"}, "--n", "64", "--order", "3", "--steps", "3", "--warmup", "2")
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 3
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 2
