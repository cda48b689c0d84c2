"""Multi-GPU plumbing of bench.py on CPU: `--gpus N` runs N independent
replicas of the workload (the path has no exchange step that one GPU per
problem would need), so the process group only carries barriers and the max
over ranks of the device times.  Two gloo ranks stand in for two GPUs."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, dist = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(dist)
        # every rank's own device time; the line reports the slowest
        t = bench.max_over_ranks(dist, 100.0 + 10.0 * rank)
        bench.barrier(dist)
        q.put((r, w, local, t, bench.whole_job_seconds_per_solve(t, w)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_max_and_report_the_whole_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == 110.0 for o in out)               # max over ranks, seen by both
    assert all(o[4] == pytest.approx(0.055) for o in out)  # 2 solves in 110 ms


def test_single_process_has_no_group():
    sys.path.insert(0, ROOT)
    import bench
    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        assert bench.dist_setup(1) == (0, 1, 0, None)
        assert bench.max_over_ranks(None, 3.5) == 3.5
        assert bench.whole_job_seconds_per_solve(712.0, 1) == pytest.approx(0.712)
    finally:
        os.environ.update(env)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "ref_small_measure", lambda *a: called.append(1))

    class A:
        warmup, steps = 3, 1
    assert bench.run_reference(A()) == 0 and not called


def test_a_failing_side_measurement_keeps_the_line():
    sys.path.insert(0, ROOT)
    import bench

    def boom(x):
        raise RuntimeError("no device %d" % x)

    assert bench.soft(lambda a, b: a + b, 2, 3) == 5
    assert bench.soft(boom, 7) == {"error": "RuntimeError: no device 7"}
    with pytest.raises(RuntimeError):
        bench.soft(boom, 7, dist=object())          # several ranks: the failure propagates
