"""One day of the pipeline split over the ranks of a torch.distributed group
(strong scaling), as the upstream splits it over GPUs, but with the exchange
done by collectives instead of P2P copies and a host relay
(main_recon_online.cu:319-356; viss_recon_kernel.cuh:740-815):

  stage 1: rank r sums all pixels for a contiguous range of time steps
           (its half-baselines); the float32 V_half pieces are all-gathered,
           so every rank holds the day's V;
  stage 2: rank r reconstructs a contiguous range of pixels (whole 1024-pixel
           blocks) from the full V; the C / W pieces are gathered to rank 0.

The arithmetic is the single-GPU kernels' (vb_viss_halfsym,
vb_phase_correct_expand, vb_recon_batched) on pointer ranges of the
pipeline's resident arrays, so the sharded day equals the single-GPU day up
to the order of FP64 partial sums.

Two ways to run the day:
  run_day_device  -- every piece stays in device memory: V pieces are
      all-gathered (NCCL) straight into a full-V device buffer that stage 2
      reads, and the C / W pieces are gathered into rank 0's device buffers;
      the collectives run on zero-copy torch views of the library's buffers
      (DeviceExchange), with no host copy of V or C on any rank;
  run_day         -- pieces are host arrays and the exchange is pluggable
      (TorchExchange over any torch.distributed backend); `compute` can be
      any object with stage1 / stage2 (the CPU tests use the FP64 oracle).
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def step_ranges(total_steps: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, balanced ranges of time steps, one per rank."""
    base, rem = divmod(total_steps, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < rem else 0)
        out.append((lo, hi))
        lo = hi
    return out


def pixel_ranges(npix: int, world: int, align: int = 1024) -> list[tuple[int, int]]:
    """Contiguous ranges of whole `align`-pixel blocks, balanced by blocks."""
    nblk = -(-npix // align)
    out = []
    for lo_b, hi_b in step_ranges(nblk, world):
        out.append((min(lo_b * align, npix), min(hi_b * align, npix)))
    return out


class TorchExchange:
    """all_gather / gather of float32 and uint32 pieces of unequal length over
    a torch.distributed group (padded to the longest piece)."""

    def __init__(self, dist, device):
        self.dist = dist
        self.device = device

    def _gather(self, piece: np.ndarray, sizes: list[int], to_all: bool, rank: int):
        import torch
        world = len(sizes)
        n = max(sizes) if sizes else 0
        pad = np.zeros(n, dtype=piece.dtype)
        pad[: piece.size] = piece
        view = pad.view(np.int32) if piece.dtype.itemsize == 4 else pad
        t = torch.from_numpy(view).to(self.device)
        bufs = [torch.empty_like(t) for _ in range(world)]
        self.dist.all_gather(bufs, t)
        if not to_all and rank != 0:
            return None
        parts = [b.cpu().numpy().view(piece.dtype)[: s] for b, s in zip(bufs, sizes)]
        return np.concatenate(parts) if parts else np.empty(0, piece.dtype)

    def all_gather(self, piece, sizes, rank):
        return self._gather(piece, sizes, True, rank)

    def gather0(self, piece, sizes, rank):
        return self._gather(piece, sizes, False, rank)


class DeviceView:
    """A range of device memory owned by this library, exposed through the CUDA
    array interface so that torch.as_tensor makes a zero-copy tensor of it."""

    def __init__(self, ptr: int, count: int, dtype):
        self.ptr, self.count, self.dtype = int(ptr), int(count), np.dtype(dtype)

    @property
    def __cuda_array_interface__(self) -> dict:
        return {"shape": (self.count,), "typestr": self.dtype.str, "data": (self.ptr, False), "version": 2}

    def tensor(self, device):
        import torch
        return torch.as_tensor(self, device=device)


class DeviceExchange:
    """Collectives on device tensors over a torch.distributed NCCL group:
    pieces of unequal length are padded to the longest in a staging tensor
    (kept across calls), exchanged, and copied device to device into the
    destination, which may alias the library's own buffers."""

    def __init__(self, dist, device):
        self.dist = dist
        self.device = device
        self._stage = {}

    def _staging(self, key: str, n: int, dtype):
        import torch
        t = self._stage.get(key)
        if t is None or t.numel() < n or t.dtype != dtype:
            t = torch.empty(n, dtype=dtype, device=self.device)
            self._stage[key] = t
        return t[:n]

    def all_gather_into(self, out, piece, sizes: list[int]) -> None:
        """out[offset_r : offset_r + sizes[r]] = rank r's piece, on every rank."""
        world = len(sizes)
        n = max(sizes)
        if all(sz == n for sz in sizes):
            self.dist.all_gather_into_tensor(out[: n * world], piece)
            return
        src = self._staging("ag_src", n, piece.dtype)
        src[: piece.numel()].copy_(piece)
        dst = self._staging("ag_dst", n * world, piece.dtype)
        self.dist.all_gather_into_tensor(dst, src)
        off = 0
        for r, sz in enumerate(sizes):
            out[off: off + sz].copy_(dst[r * n: r * n + sz])
            off += sz

    def gather0_into(self, out, piece, sizes: list[int], rank: int) -> None:
        """Rank 0: out[offset_r : offset_r + sizes[r]] = rank r's piece; the
        other ranks only send (out may be None there)."""
        world = len(sizes)
        n = max(sizes)
        src = piece if piece.numel() == n else self._staging("g_src", n, piece.dtype)
        if src is not piece:
            src[: piece.numel()].copy_(piece)
        if rank == 0:
            dst = self._staging("g_dst", n * world, piece.dtype)
            self.dist.gather(src, gather_list=list(dst.view(world, n).unbind(0)), dst=0)
            off = 0
            for r, sz in enumerate(sizes):
                out[off: off + sz].copy_(dst[r * n: r * n + sz])
                off += sz
        else:
            self.dist.gather(src, gather_list=None, dst=0)


class GpuCompute:
    """The library's kernels on pointer ranges of a vb.Pipeline's arrays."""

    def __init__(self, vb, p):
        self.vb, self.p = vb, p
        L = vb.lib()
        self.L = L
        cfg = p.cfg
        self.sky = vb.Sky()
        self.sky.npix = p.npix
        for k in ("B", "l", "m", "n", "cx", "cy", "cz", "cosA", "sinA"):
            setattr(self.sky, k, p.ptr(k)[0])
        self.sky.tile_pix = cfg.viss_tile_pix
        self.keys = ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2", "cosphi1", "cosphi2")
        self.base = {k: p.ptr(k)[0] for k in self.keys}
        rep = p.run()   # resident single-GPU day: sets up the pipeline (and its automatic bl_max)
        self.o1 = vb.Stage1Opts(precision=cfg.precision, cull=cfg.cull, phase_corrected=1, blockage=cfg.blockage,
                                bpt=cfg.stage1_bpt, stage_pix=cfg.stage1_stage_pix,
                                ctas_per_sm=cfg.stage1_ctas_per_sm, items_per_cta=cfg.stage1_items_per_cta,
                                refine_pix=cfg.stage1_refine_pix)
        self.o2 = vb.Stage2Opts(mirror=cfg.mirror, blockage=cfg.blockage, occ_mode=cfg.occ_mode,
                                precision=cfg.precision, cull=cfg.stage2_cull, grid_res=cfg.grid_res,
                                bl_max=rep["bl_max_m"], lambda_=cfg.lambda_m, ppt=cfg.stage2_ppt,
                                items_per_cta=cfg.stage2_items_per_cta)

    def _buf(self, name: str, nbytes: int):
        """Device buffer `name` of at least `nbytes`, kept across calls."""
        if not hasattr(self, "_bufs"):
            self._bufs = {}
        b = self._bufs.get(name)
        if b is None or b.nbytes < nbytes:
            if b is not None:
                b.free()
            b = self.vb.DeviceBuffer(nbytes)
            self._bufs[name] = b
        return b

    def baselines(self, lo: int, hi: int):
        p, vb = self.p, self.vb
        b = vb.Baselines()
        b.n_full, b.nbl, b.cosphi = 2 * p.nbl * (hi - lo), p.nbl, p.cosphi
        off = 4 * 2 * p.nbl * lo
        for k in self.keys:
            if self.base[k]:
                setattr(b, k, self.base[k] + off)
        return b

    def stage1(self, lo: int, hi: int) -> np.ndarray:
        """float32 (re, im) V_half of the half-baselines of steps [lo, hi)."""
        vb, L = self.vb, self.L
        if hi <= lo:
            return np.empty(0, np.float32)
        b = self.baselines(lo, hi)
        nh = b.n_full // 2
        need = L.vb_stage1_workspace_bytes(C.byref(self.sky), C.byref(b), C.byref(self.o1))
        ws, Vd, Vh = self._buf("ws1", need), self._buf("Vd", 16 * nh), self._buf("Vh", 8 * nh)
        vb.check(L.vb_viss_halfsym(C.byref(self.sky), C.byref(b), C.byref(self.o1), ws.ptr, ws.nbytes, Vd.ptr,
                                   None, None))
        vb.check(L.vb_phase_correct_expand(Vd.ptr, b.w, nh, b.nbl, 1, Vh.ptr, None, None))
        return Vh.to_array(np.float32, 2 * nh)

    def stage2(self, V_half: np.ndarray, plo: int, phi: int):
        """C (float32) and W (uint32) of pixels [plo, phi) from the full V_half."""
        vb, L, p = self.vb, self.L, self.p
        n = phi - plo
        if n <= 0:
            return np.empty(0, np.float32), np.empty(0, np.uint32)
        sky = vb.Sky()
        sky.npix = n
        for k in ("l", "m", "n"):
            setattr(sky, k, getattr(self.sky, k) + 4 * plo)
        sky.B = self.sky.B + 4 * plo
        bl = self.baselines(0, p.n_half // p.nbl)
        need = L.vb_stage2_workspace_bytes(p.n_half, p.nseg, n, C.byref(self.o2))
        Vh = np.ascontiguousarray(V_half, np.float32)
        ws, dV = self._buf("ws2", need), self._buf("V", Vh.nbytes)
        vb.check(L.vb_memcpy(dV.ptr, Vh.ctypes.data, Vh.nbytes, 0))
        Cb, Wb = self._buf("C", 4 * n), self._buf("W", 4 * n)
        vb.check(L.vb_recon_batched(C.byref(sky), C.byref(bl), dV.ptr, p.nseg, p.ptr("seg_t0")[0],
                                    p.ptr("seg_tlen")[0], C.byref(self.o2), ws.ptr, ws.nbytes, Cb.ptr, Wb.ptr, None,
                                    None, None))
        return Cb.to_array(np.float32, n), Wb.to_array(np.uint32, n)


    # --- device-resident pieces (run_day_device) -----------------------------
    def full_buffers(self, device) -> dict:
        """Zero-copy tensors of the day-sized device buffers: V (float32 (re, im)
        per half-baseline), C (float32) and W (as int32) per pixel."""
        p = self.p
        V = self._buf("V_full", 8 * p.n_half)
        Cb, Wb = self._buf("C_full", 4 * p.npix), self._buf("W_full", 4 * p.npix)
        return {"V": DeviceView(V.ptr, 2 * p.n_half, np.float32).tensor(device),
                "C": DeviceView(Cb.ptr, p.npix, np.float32).tensor(device),
                "W": DeviceView(Wb.ptr, p.npix, np.int32).tensor(device), "V_ptr": V.ptr}

    def stage1_device(self, lo: int, hi: int, device):
        """Tensor view of the float32 (re, im) V_half of steps [lo, hi), left in
        device memory."""
        vb, L = self.vb, self.L
        b = self.baselines(lo, hi)
        nh = b.n_full // 2
        need = L.vb_stage1_workspace_bytes(C.byref(self.sky), C.byref(b), C.byref(self.o1))
        ws, Vd, Vh = self._buf("ws1", need), self._buf("Vd", 16 * max(nh, 1)), self._buf("Vh", 8 * max(nh, 1))
        if nh > 0:
            vb.check(L.vb_viss_halfsym(C.byref(self.sky), C.byref(b), C.byref(self.o1), ws.ptr, ws.nbytes, Vd.ptr,
                                       None, None))
            vb.check(L.vb_phase_correct_expand(Vd.ptr, b.w, nh, b.nbl, 1, Vh.ptr, None, None))
        return DeviceView(Vh.ptr, 2 * nh, np.float32).tensor(device)

    def stage2_device(self, V_ptr: int, plo: int, phi: int, device):
        """Tensor views of C (float32) and W (int32) of pixels [plo, phi),
        reconstructed from the full V already in device memory at V_ptr."""
        vb, L, p = self.vb, self.L, self.p
        n = phi - plo
        Cb, Wb = self._buf("C", 4 * max(n, 1)), self._buf("W", 4 * max(n, 1))
        if n > 0:
            sky = vb.Sky()
            sky.npix = n
            for k in ("l", "m", "n"):
                setattr(sky, k, getattr(self.sky, k) + 4 * plo)
            sky.B = self.sky.B + 4 * plo
            bl = self.baselines(0, p.n_half // p.nbl)
            need = L.vb_stage2_workspace_bytes(p.n_half, p.nseg, n, C.byref(self.o2))
            ws = self._buf("ws2", need)
            vb.check(L.vb_recon_batched(C.byref(sky), C.byref(bl), V_ptr, p.nseg, p.ptr("seg_t0")[0],
                                        p.ptr("seg_tlen")[0], C.byref(self.o2), ws.ptr, ws.nbytes, Cb.ptr, Wb.ptr,
                                        None, None, None))
        return (DeviceView(Cb.ptr, n, np.float32).tensor(device), DeviceView(Wb.ptr, n, np.int32).tensor(device))


def run_day_device(compute: GpuCompute, exchange: DeviceExchange, rank: int, world: int, total_steps: int,
                   nbl: int, npix: int, device):
    """The sharded day with every piece in device memory.  Returns device
    tensors (V, C, W): V (float32 (re, im) of all half-baselines) on every
    rank; C (float32) and W (int32 view of the uint32 counts) complete on rank
    0 only.  They alias the compute object's buffers (valid until its next day)."""
    full = compute.full_buffers(device)
    steps = step_ranges(total_steps, world)
    lo, hi = steps[rank]
    V_piece = compute.stage1_device(lo, hi, device)
    exchange.all_gather_into(full["V"], V_piece, [2 * nbl * (h - l) for l, h in steps])
    pix = pixel_ranges(npix, world)
    plo, phi = pix[rank]
    C_piece, W_piece = compute.stage2_device(full["V_ptr"], plo, phi, device)
    sizes = [h - l for l, h in pix]
    exchange.gather0_into(full["C"] if rank == 0 else None, C_piece, sizes, rank)
    exchange.gather0_into(full["W"] if rank == 0 else None, W_piece, sizes, rank)
    return full["V"], full["C"], full["W"]


def run_day(compute, exchange, rank: int, world: int, total_steps: int, nbl: int, npix: int):
    """The sharded day: returns (V_half, C, W) on rank 0 (V_half on every
    rank), (V_half, None, None) on the others."""
    steps = step_ranges(total_steps, world)
    lo, hi = steps[rank]
    V_piece = compute.stage1(lo, hi)
    V_half = exchange.all_gather(V_piece, [2 * nbl * (h - l) for l, h in steps], rank)
    pix = pixel_ranges(npix, world)
    plo, phi = pix[rank]
    C_piece, W_piece = compute.stage2(V_half, plo, phi)
    sizes = [h - l for l, h in pix]
    Cfull = exchange.gather0(C_piece, sizes, rank)
    Wfull = exchange.gather0(W_piece, sizes, rank)
    return V_half, Cfull, Wfull
