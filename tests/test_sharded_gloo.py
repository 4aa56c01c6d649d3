"""The strong-scaling split of one day over ranks (viss_optimize_ws_b200/
sharded.py): stage 1 by time-step ranges with an all-gather of V, stage 2 by
pixel ranges with a gather of C / W to rank 0.  World size 2 over gloo on
CPU, the FP64 oracle standing in for the GPU kernels: the sharded day equals
the single-process day bit for bit (every term's arithmetic is range
independent)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from viss_optimize_ws_b200 import sharded

NSIDE, NSAT, T, SEGS = 8, 4, 12, 3


def test_partitions_cover_exactly():
    for total, world in ((12, 2), (13, 4), (3, 4), (1024, 8)):
        r = sharded.step_ranges(total, world)
        assert r[0][0] == 0 and r[-1][1] == total and all(r[i][1] == r[i + 1][0] for i in range(world - 1))
        assert max(h - l for l, h in r) - min(h - l for l, h in r) <= 1
    for npix, world in ((768, 2), (786432, 8), (3072, 3), (1000, 4)):
        r = sharded.pixel_ranges(npix, world)
        assert r[0][0] == 0 and r[-1][1] == npix and all(r[i][1] == r[i + 1][0] for i in range(world - 1))
        assert all(l % 1024 == 0 or l == npix for l, _ in r)


class OracleCompute:
    """CPU stand-in for GpuCompute with the same two methods."""

    def __init__(self):
        from oracle import py as orp
        self.orp = orp
        npix = 12 * NSIDE * NSIDE
        l, m, n = (a.astype(np.float32) for a in orp.nest_lmn_f64(NSIDE))
        B = (orp.make_sky(NSIDE, 3).astype(np.float64) * (4 * np.pi / npix)).astype(np.float32)
        self.sky = dict(B=B, l=l, m=m, n=n)
        self.bl = orp.syn_baselines(NSAT, T, lam=30.0)
        self.bl["cosphi"] = float(-np.sqrt(1 - (6371.0 / 6871.0) ** 2))
        self.nbl = self.bl["nbl"]
        self.npix = npix
        self.t0 = np.array([0, 4, 8], np.int32)
        self.tl = np.array([4, 4, 4], np.int32)

    def _bl(self, lo, hi):
        i0, i1 = 2 * self.nbl * lo, 2 * self.nbl * hi
        b = {k: np.ascontiguousarray(v[i0:i1]) for k, v in self.bl.items() if isinstance(v, np.ndarray)}
        b["nbl"], b["cosphi"] = self.nbl, self.bl["cosphi"]
        return b

    def stage1(self, lo, hi):
        if hi <= lo:
            return np.empty(0, np.float32)
        return self.orp.stage1(self.sky, self._bl(lo, hi), phase_corrected=1, precision=1).astype(np.float32)

    def stage2(self, V_half, plo, phi):
        sky = {k: np.ascontiguousarray(v[plo:phi]) for k, v in self.sky.items()}
        Cc, W, _ = self.orp.stage2(sky, self.bl, V_half, self.t0, self.tl, mirror=1, blockage=1, occ_mode=2,
                                   bl_max=200e3, lam=30.0, grid_res=65, precision=1)
        return Cc.astype(np.float32), W


class LocalExchange:
    def all_gather(self, piece, sizes, rank):
        return piece

    def gather0(self, piece, sizes, rank):
        return piece


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import datetime

    import torch
    import torch.distributed as td
    try:
        td.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
        comp = OracleCompute()
        ex = sharded.TorchExchange(td, torch.device("cpu"))
        V, Cc, W = sharded.run_day(comp, ex, rank, ws, T, comp.nbl, comp.npix)
        q.put((rank, "ok", V, Cc, W))
        td.destroy_process_group()
    except Exception as e:
        q.put((rank, "error", repr(e)[:300], None, None))


def test_sharded_day_equals_single_process():
    comp = OracleCompute()
    V1, C1, W1 = sharded.run_day(comp, LocalExchange(), 0, 1, T, comp.nbl, comp.npix)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=180) for _ in range(2)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert [o[1] for o in out] == ["ok", "ok"], out
    for rank, _, V, Cc, W in out:
        assert np.array_equal(V.view(np.uint32), V1.view(np.uint32))
        if rank == 0:
            assert np.array_equal(Cc.view(np.uint32), C1.view(np.uint32))
            assert np.array_equal(W, W1)
        else:
            assert Cc is None and W is None
    assert (W1 > 0).any()


class OracleDeviceCompute(OracleCompute):
    """CPU stand-in for GpuCompute's device-resident methods: the same pieces
    as CPU torch tensors, so that run_day_device and DeviceExchange run their
    collective steps over gloo."""

    def full_buffers(self, device):
        import torch
        self._full = {"V": torch.zeros(2 * self.nbl * T, dtype=torch.float32),
                      "C": torch.zeros(self.npix, dtype=torch.float32),
                      "W": torch.zeros(self.npix, dtype=torch.int32)}
        return dict(self._full, V_ptr=None)

    def stage1_device(self, lo, hi, device):
        import torch
        return torch.from_numpy(self.stage1(lo, hi).copy())

    def stage2_device(self, V_ptr, plo, phi, device):
        import torch
        Cc, W = self.stage2(self._full["V"].numpy(), plo, phi)
        return torch.from_numpy(Cc.copy()), torch.from_numpy(W.astype(np.int32))


def _worker_device(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import datetime

    import torch
    import torch.distributed as td
    try:
        td.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
        ex = sharded.DeviceExchange(td, torch.device("cpu"))
        # unequal pieces: rank r contributes r + 2 values r*100 + i
        sizes = [r + 2 for r in range(ws)]
        piece = torch.tensor([rank * 100 + i for i in range(sizes[rank])], dtype=torch.float32)
        out = torch.full((sum(sizes),), -1.0)
        ex.all_gather_into(out, piece, sizes)
        g = torch.full((sum(sizes),), -1.0) if rank == 0 else None
        ex.gather0_into(g, piece, sizes, rank)
        comp = OracleDeviceCompute()
        V, Cc, W = sharded.run_day_device(comp, ex, rank, ws, T, comp.nbl, comp.npix, torch.device("cpu"))
        q.put((rank, "ok", out.numpy(), None if g is None else g.numpy(), V.numpy().copy(),
               Cc.numpy().copy() if rank == 0 else None, W.numpy().copy() if rank == 0 else None))
        td.destroy_process_group()
    except Exception as e:
        q.put((rank, "error", repr(e)[:300], None, None, None, None))


def test_device_exchange_and_day_over_two_ranks():
    """DeviceExchange (padded all-gather into a destination, gather to rank 0
    only) with unequal pieces, and run_day_device with the oracle standing in
    for the kernels: world size 2 over gloo equals the single-process day bit
    for bit; C and W are complete on rank 0."""
    comp = OracleCompute()
    V1, C1, W1 = sharded.run_day(comp, LocalExchange(), 0, 1, T, comp.nbl, comp.npix)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker_device, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=180) for _ in range(2)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert [o[1] for o in out] == ["ok", "ok"], out
    expect = np.array([0, 1, 100, 101, 102], np.float32)
    for rank, _, ag, g, V, Cc, W in out:
        assert np.array_equal(ag, expect)
        assert np.array_equal(V.view(np.uint32), V1.view(np.uint32))
        if rank == 0:
            assert np.array_equal(g, expect)
            assert np.array_equal(Cc.view(np.uint32), C1.view(np.uint32))
            assert np.array_equal(W.astype(np.uint32), W1)
        else:
            assert g is None
