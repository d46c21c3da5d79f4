"""bench.py's multi-GPU plumbing on the CPU: replicas report the slowest
rank's time and the units of all ranks (two gloo ranks), and `--gpus N`
without an outside launcher re-runs the script under torch.distributed.run
with one process per GPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = 10.0 * (rank + 1)          # rank 1 is the slow one
        ms, rate = bench.aggregate_rate(ms_local, world, 60, dist, "cpu")
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as fh:
            fh.write(f"{ms} {rate}")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank(tmp_path):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        ms, rate = map(float, open(tmp_path / f"r{r}.txt").read().split())
        assert ms == 20.0
        assert rate == pytest.approx(2 * 60 / 0.020)


def test_single_process_reports_its_own_time():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_rate(25.0, 1, 60) == (25.0, pytest.approx(2400.0))


def test_gpus_flag_launches_one_replica_per_gpu(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    seen = {}

    class Done:
        returncode = 0

    def fake_run(cmd, *a, **k):
        seen["cmd"] = cmd
        return Done()

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    argv = ["--gpus", "4", "--steps", "2", "--warmup", "3"]
    assert bench.main(argv) == 0
    cmd = seen["cmd"]
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd
    assert cmd[-len(argv):] == argv and cmd[-len(argv) - 1].endswith("bench.py")
