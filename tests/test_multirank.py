"""The N>1 bench path on CPU: world_size-2 gloo ranks launched the way the
bench is launched (torch.distributed.run, 127.0.0.1), checking that the job
time is the max over ranks, that the whole-job value aggregates the replicas,
and that the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reduce_max_and_aggregate(tmp_path):
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "tests" / "_multirank_worker.py"), str(tmp_path)]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    for k, g in enumerate(got):
        assert g["rank"] == k and g["world"] == 2 and g["local"] == k
        assert g["dev_s"] == pytest.approx(2.0)   # rank 1's 2 s, seen by both ranks
        assert g["e2e_s"] == pytest.approx(0.5)   # rank 0's 0.5 s, seen by both ranks
        assert g["value"] == pytest.approx(2.0)   # 2 x 2 M units in 2 s = 2 M units/s


def test_helpers_without_process_group():
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.whole_job_rate(132_710_400, 1, 1.0) == pytest.approx(132.7104)
    assert bench.whole_job_rate(132_710_400, 8, 2.0) == pytest.approx(530.8416)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), {"steps": 1, "warmup": 3, "cpu_spp": 1})()
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
