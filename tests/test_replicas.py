"""The multi-GPU plumbing of bench.py (vikalp_b200.replicas): replicas with no
collective on the data path, a barrier around the timed region, the job's
time as the slowest rank's and its rate as all ranks' units over that time.
Run here as two gloo ranks on the CPU (torch.multiprocessing, spawn)."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from vikalp_b200 import replicas
    r = replicas.init(backend="gloo", timeout_s=60)
    assert (r.world, r.rank, r.device) == (world, rank, "cpu")
    replicas.barrier(r)
    # rank k processed 100 * (k + 1) units in 1 + k seconds
    rate, t = replicas.whole_job_rate(r, 100.0 * (rank + 1), 1.0 + rank)
    mx = replicas.max_over_ranks(r, 5.0 - rank)
    out[rank] = (rate, t, mx)
    replicas.finish(r)


@pytest.mark.parametrize("world", [2, 3])
def test_replica_reductions_over_gloo_ranks(world):
    port = _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    total = sum(100.0 * (k + 1) for k in range(world))
    slowest = 1.0 + (world - 1)
    for k in range(world):
        rate, t, mx = out[k]
        assert t == slowest and mx == 5.0  # every rank sees the same job-level figures
        assert rate == pytest.approx(total / slowest)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from vikalp_b200 import replicas
    r = replicas.init()
    assert r.world == 1 and r.backend is None
    assert replicas.whole_job_rate(r, 640, 2.0) == (320.0, 2.0)
    replicas.barrier(r)
    replicas.finish(r)
