"""bench.py --gpus N starts its own N ranks (one process per GPU) when it is
not already running under torch.distributed.run, and refuses a rank count
that differs from --gpus.  Checked on CPU through the same launcher with the
gloo backend and the --launch-check mode (process group only, no kernels)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _env():
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    return env


def test_gpus_2_starts_two_ranks():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--dist-backend", "gloo", "--launch-check"],
                       capture_output=True, text=True, timeout=240, env=_env(), cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["launch_check"] and d["n_gpus"] == 2 and d["ranks_joined"] == 2


def test_rank_count_must_match_gpus():
    env = _env()
    env.update({"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--launch-check"], capture_output=True, text=True, timeout=120,
                       env=env, cwd=ROOT)
    assert r.returncode != 0
    assert "--gpus 2 but 1 ranks" in r.stderr
