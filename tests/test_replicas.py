"""The multi-GPU plumbing of bench.py (replicas over events, no data-path
collective) on two gloo ranks on the CPU: barrier, max / sum reductions and
the whole-job rate (all ranks' events over the slowest rank's time)."""
import os
import pathlib
import socket
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT / "freestream-milne_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from replicas import Replicas
    r = Replicas(backend="gloo", timeout_s=30)
    r.barrier()
    res = {"seed": r.seed(3), "max": r.max(1.5 + rank), "sum": r.sum(10 * (rank + 1)),
           "rate": r.rate(100, 2.0 + rank)}
    r.close()
    out.put((rank, res))


def test_two_gloo_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0]["seed"] == 3 and got[1]["seed"] == 1003
    for k in (0, 1):
        assert got[k]["max"] == 2.5
        assert got[k]["sum"] == 30
        assert got[k]["rate"] == pytest.approx(200 / 3.0)


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT / "freestream-milne_b200"))
    from replicas import Replicas
    old = {k: os.environ.pop(k, None) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        r = Replicas()
        assert r.world == 1 and r.max(3.0) == 3.0 and r.rate(50, 2.0) == 25.0
        r.close()
    finally:
        for k, v in old.items():
            if v is not None:
                os.environ[k] = v
