"""The multi-rank bench plumbing on CPU with gloo, world size 2: every rank
reports its own device time, rank 0's number is the max over ranks, and the
whole-job value counts the particles of all replicas (the step itself does
not shard: ranks are independent replicas with no data-path collective)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    r, w, loc = bench.dist_env()
    my_ms = 10.0 + 5.0 * rank
    t = bench.max_over_ranks(my_ms, "cpu")
    v = bench.replica_value(w, 1000, 4, t)
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, loc, t, v))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    for r, w, loc, t, v in out:
        assert t == 15.0                          # the slower rank's time on every rank
        assert v == pytest.approx(2 * 1000 * 4 / 15e-3)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), dict(mc3d="literal", steps=1, warmup=3))()
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
