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
