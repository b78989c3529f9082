"""bench.py's process layout, without a GPU: `--gpus N` starts N ranks of itself (under
torch.distributed.run on 127.0.0.1), and a torchrun world that disagrees with --gpus is refused."""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def _env(**kw):
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env.update(kw)
    return env


def test_gpus_two_starts_two_ranks():
    r = subprocess.run([sys.executable, BENCH, "--gpus", "2", "--probe-ranks"],
                       capture_output=True, text=True, timeout=300, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in re.findall(r"\{[^{}]*\}", r.stdout)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    assert all(x["world"] == 2 and x["gpus"] == 2 for x in lines)
    assert sorted(x["local_rank"] for x in lines) == [0, 1]


def test_single_gpu_runs_in_process():
    r = subprocess.run([sys.executable, BENCH, "--probe-ranks"], capture_output=True, text=True,
                       timeout=120, env=_env())
    assert r.returncode == 0
    assert json.loads(r.stdout.strip().splitlines()[-1]) == {"rank": 0, "world": 1,
                                                             "local_rank": 0, "gpus": 1}


def test_world_size_mismatch_is_refused():
    r = subprocess.run([sys.executable, BENCH, "--gpus", "4", "--probe-ranks"],
                       capture_output=True, text=True, timeout=120,
                       env=_env(WORLD_SIZE="2", RANK="0", LOCAL_RANK="0"))
    assert r.returncode == 2
    assert "WORLD_SIZE=2" in r.stderr
