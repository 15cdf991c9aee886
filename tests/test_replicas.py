"""Multi-GPU replica plumbing on CPU: two gloo ranks (world size 2) take the
same collective steps as bench.py's GPU ranks -- barrier, max over ranks of
each timed duration -- and the whole-job rate is every rank's work over the
slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from unitywindsimulation_b200.replicas import ReplicaGroup, deal, env_ranks, whole_job_rate


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


def test_deal_covers_every_case_once_and_balances_the_load():
    from unitywindsimulation_b200 import cases
    sizes = [c.n_cells for c in cases.batch_directions()]
    for world in (1, 2, 3, 4, 8):
        parts = deal(sizes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # largest-first onto the least-loaded rank: the heaviest rank carries
        # at most the mean plus one case
        assert max(loads) <= sum(sizes) / world + max(sizes)
    assert deal([5, 3, 3], 2) == [[0], [1, 2]]
    assert deal([1, 2], 4) == [[1], [0], [], []]
    with pytest.raises(ValueError):
        deal([1], 0)


def _deal_rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sizes = [9, 7, 6, 5, 4, 2, 1]
    g = ReplicaGroup("gloo", timeout_s=60)
    mine = deal(sizes, g.world)[g.rank]
    g.barrier()
    # each rank "takes" one ms per size unit of its share; the whole job waits
    # for the slowest rank
    ms_max = g.max_over_ranks(float(sum(sizes[i] for i in mine)))
    g.close()
    out.put((rank, mine, ms_max))


def test_two_gloo_ranks_step_disjoint_shares_of_the_cases():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_deal_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0), (r1, m1, t1) = res
    assert sorted(m0 + m1) == list(range(7)) and not set(m0) & set(m1)
    assert t0 == t1 == 17.0  # loads 17 and 17: 9+5+2+1 and 7+6+4
