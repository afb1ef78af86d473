"""bench.py's rank launch, on CPU: `--gpus N` without a launcher re-runs the
script under torch.distributed.run with N ranks, and rank 0 reports the
aggregate over all of them. The `--stand-in` switch swaps the GPU step for a
small numpy step on gloo ranks, so only the launch and the aggregation run
here; the GPU arm shares both (_init_dist, _reduce, relaunch)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    env.pop("RANK", None)
    env.pop("LOCAL_RANK", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--stand-in", "--steps", "2", *args],
                       capture_output=True, text=True, timeout=240, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    return json.loads(lines[0])


@pytest.mark.parametrize("mode,scaling", [("replicas", "weak"), ("sharded", "strong")])
def test_gpus_flag_launches_that_many_ranks(mode, scaling):
    d = _run("--gpus", "2", "--mode", mode)
    assert d["n_gpus"] == 2
    assert d["scaling"] == scaling
    assert d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0


def test_single_rank_runs_in_process():
    d = _run("--gpus", "1")
    assert d["n_gpus"] == 1
