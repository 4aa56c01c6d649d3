"""The N>1 path of bench.py (independent replicas, barrier + max-over-ranks
timing) as world_size-2 gloo process groups on CPU; and a rank that fails
before the barrier: the other rank's collective ends with an error instead
of hanging (failure detected on the host, no GPU involved)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    try:
        d = bench.Dist(ws, rank, backend="gloo", timeout_s=8.0)
        if rank == fail_rank:
            raise RuntimeError("injected failure before the barrier")
        d.barrier()
        t = [10.0, 12.5, 11.0, 9.0][rank]
        m = d.max(t)
        v = bench.replica_value(1e9, 4, m, ws)
        q.put((rank, "ok", m, v))
        d.close()
    except Exception as e:  # report instead of hanging
        q.put((rank, "error", type(e).__name__, str(e)[:200]))


def run(ws, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q, fail_rank)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_replicas_max_over_ranks():
    out = run(2)
    assert [o[1] for o in out] == ["ok", "ok"]
    for _, _, m, v in out:
        assert m == 12.5
        assert v == pytest.approx(2 * 1e9 * 4 / 12.5e-3 / 1e9)


def test_rank_failure_is_reported_not_hung():
    out = run(2, fail_rank=1)
    states = {o[0]: o[1] for o in out}
    assert states[1] == "error"
    assert states[0] == "error"       # the surviving rank's barrier ends with an error


def test_each_rank_builds_its_pipeline_on_its_own_gpu(vb):
    """Under torchrun every rank's pipeline must name its LOCAL_RANK device: the
    library selects the configured device on every call, so a config left at
    the default would put every rank on GPU 0."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    for local in (0, 3, 7):
        kw = bench.rank_workload_kwargs(local)
        assert kw["device"] == local
        assert vb.run_config(**kw).device == local
        assert {k: v for k, v in kw.items() if k != "device"} == bench.config_kwargs(bench.HEADLINE)
    assert bench.rank_workload_kwargs(5, "fp64")["precision"] == "fp64"
