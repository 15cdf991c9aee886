"""Multi-GPU replica plumbing on CPU: two gloo ranks (world size 2) take the
same collective steps as bench.py's GPU ranks -- barrier, max over ranks of
each timed duration -- and the whole-job rate is every rank's work over the
slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from unitywindsimulation_b200.replicas import ReplicaGroup, env_ranks, whole_job_rate


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    g = ReplicaGroup("gloo", timeout_s=60)
    assert (g.rank, g.world, g.local) == (rank, world, rank)
    g.barrier()
    ms = 10.0 * (rank + 1)            # rank 1 is the slow one
    ms_max = g.max_over_ranks(ms)
    e_ms = g.max_over_ranks(5.0 + rank)
    rate = whole_job_rate(1000, 4, ms_max, g.world)
    g.close()
    out.put((rank, ms_max, e_ms, rate))


def test_two_gloo_ranks_agree_on_max_and_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms_max, e_ms, rate in res:
        assert ms_max == 20.0 and e_ms == 6.0
        # 2 ranks x 1000 cells x 4 steps in 20 ms
        assert rate == pytest.approx(2 * 1000 * 4 / 0.020 / 1e6)


def test_single_process_is_rank_zero_of_one(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert env_ranks() == (0, 1, 0)
    g = ReplicaGroup("gloo")
    assert not g.dist and g.max_over_ranks(3.5) == 3.5
    g.barrier()
    g.close()


def test_rate_rejects_zero_time():
    with pytest.raises(ValueError):
        whole_job_rate(10, 1, 0.0, 1)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.main() == 0
    assert capsys.readouterr().out == ""
