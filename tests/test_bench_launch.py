"""bench.py --gpus N: the launch decision, and an N = 2 run of the reference arm on CPU that
reports n_gpus = 2 (the bench re-executes itself under torch.distributed.run)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_launch_plan():
    assert bench.launch_plan(1, {}) == "run"
    assert bench.launch_plan(2, {}) == "spawn"
    assert bench.launch_plan(4, {"WORLD_SIZE": "4"}) == "run"
    assert bench.launch_plan(1, {"WORLD_SIZE": "1"}) == "run"
    with pytest.raises(SystemExit):
        bench.launch_plan(8, {"WORLD_SIZE": "1"})
    with pytest.raises(SystemExit):
        bench.launch_plan(1, {"WORLD_SIZE": "2"})
    with pytest.raises(SystemExit):
        bench.launch_plan(0, {})


def test_spawn_command():
    cmd = bench.spawn_command(["--gpus", "2", "--steps", "3"], 2, 29555)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=2" in cmd and "--master-addr=127.0.0.1" in cmd and "--master-port=29555" in cmd
    assert cmd[-4:] == ["--gpus", "2", "--steps", "3"]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so")), reason="reference checker not built")
def test_reference_arm_two_ranks_reports_two_gpus():
    env = dict(os.environ, SHHD_REF_BUDGET_S="0.5", OMP_NUM_THREADS="2")
    env.pop("WORLD_SIZE", None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, out.stdout  # rank 0 alone prints
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
