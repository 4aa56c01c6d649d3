"""The strong-scaling split of one day (viss_optimize_ws_b200/sharded.py)
with the real kernels: two ranks as two processes that share this GPU and
exchange V and C over gloo on the host (their kernels never wait on each
other); the sharded day equals the single-GPU day to FP32 summation
rounding, with identical visible-group counts.  A second test runs the
device-resident day as one rank over NCCL (V and C never leave device
memory), the exchange a multi-GPU run uses."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import rel_err

pytestmark = pytest.mark.gpu

KW = dict(nside=32, orbit_model=1, nsat=8, tsteps=96, segs=3, lambda_m=30.0, occ_R_m=6371e3, cull="tilecone",
          viss_tile_pix=1024, mirror=1, grid_res=129, bl_max_m=0.0)


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch
    import torch.distributed as td
    import viss_optimize_ws_b200 as vb
    from viss_optimize_ws_b200 import sharded
    try:
        td.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
        with vb.Pipeline(vb.run_config(**KW)) as p:
            p.set_sky(vb.synthetic_sky(32, seed=8))
            p.make_baselines()
            comp = sharded.GpuCompute(vb, p)
            ex = sharded.TorchExchange(td, torch.device("cpu"))
            V, Cc, W = sharded.run_day(comp, ex, rank, ws, p.n_half // p.nbl, p.nbl, p.npix)
        q.put((rank, "ok", V, Cc, W))
        td.destroy_process_group()
    except Exception as e:
        q.put((rank, "error", repr(e)[:300], None, None))


class NoHostCopy:
    """The library handle with every host<->device copy refused: what the
    device-resident day must never do."""

    def __init__(self, L):
        self._L = L

    def __getattr__(self, name):
        f = getattr(self._L, name)
        if name == "vb_memcpy":
            def guarded(dst, src, n, kind):
                if kind != 2:
                    raise AssertionError(f"host copy of {n} bytes during the device-resident day")
                return f(dst, src, n, kind)
            return guarded
        return f


def _worker_nccl(port, q):
    """One rank over NCCL, every piece in device memory (run_day_device): the
    exchange path a multi-GPU run takes, on the one GPU this test has (a
    one-rank collective is a device copy).  Host copies of V or C are refused
    while the day runs."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch
    import torch.distributed as td
    import viss_optimize_ws_b200 as vb
    from viss_optimize_ws_b200 import sharded
    try:
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        td.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                              device_id=dev)
        with vb.Pipeline(vb.run_config(**KW)) as p:
            p.set_sky(vb.synthetic_sky(32, seed=8))
            p.make_baselines()
            comp = sharded.GpuCompute(vb, p)
            ex = sharded.DeviceExchange(td, dev)
            comp.L = NoHostCopy(comp.L)
            to_array = vb.DeviceBuffer.to_array
            vb.DeviceBuffer.to_array = lambda *a, **k: (_ for _ in ()).throw(AssertionError("download"))
            try:
                for _ in range(2):
                    Vt, Ct, Wt = sharded.run_day_device(comp, ex, 0, 1, p.n_half // p.nbl, p.nbl, p.npix, dev)
                torch.cuda.synchronize()
            finally:
                vb.DeviceBuffer.to_array = to_array
            V, Cc, W = Vt.cpu().numpy(), Ct.cpu().numpy(), Wt.cpu().numpy().view(np.uint32)
        td.destroy_process_group()
        q.put(("ok", V, Cc, W))
    except Exception as e:
        q.put(("error", repr(e)[:300], None, None))


def test_sharded_day_matches_single_gpu(gpu, vb):
    with vb.Pipeline(vb.run_config(**KW)) as p:
        p.set_sky(vb.synthetic_sky(32, seed=8))
        p.make_baselines()
        p.run()
        V1, C1, W1 = p.get("V_half"), p.get("C"), p.get("W")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    out = sorted([q.get(timeout=300) for _ in range(2)], key=lambda o: o[0])
    for pr in procs:
        pr.join(timeout=60)
        if pr.is_alive():
            pr.kill()
    assert [o[1] for o in out] == ["ok", "ok"], out
    _, _, V, Cc, W = out[0]
    assert rel_err(V, V1)[0] < 1e-6 and rel_err(Cc, C1)[0] < 1e-6
    assert np.array_equal(W, W1)
    assert np.array_equal(out[1][2].view(np.uint32), V.view(np.uint32))


def test_sharded_day_over_nccl_one_rank(gpu, vb):
    with vb.Pipeline(vb.run_config(**KW)) as p:
        p.set_sky(vb.synthetic_sky(32, seed=8))
        p.make_baselines()
        p.run()
        V1, C1, W1 = p.get("V_half"), p.get("C"), p.get("W")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pr = ctx.Process(target=_worker_nccl, args=(free_port(), q))
    pr.start()
    out = q.get(timeout=300)
    pr.join(timeout=60)
    if pr.is_alive():
        pr.kill()
    assert out[0] == "ok", out
    _, V, Cc, W = out
    assert rel_err(V, V1)[0] < 1e-6 and rel_err(Cc, C1)[0] < 1e-6
    assert np.array_equal(W, W1)
