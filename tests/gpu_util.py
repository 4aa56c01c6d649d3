"""Device-array helpers and shared fixtures data for the GPU tests."""
from __future__ import annotations

import ctypes as C

import numpy as np

import viss_optimize_ws_b200 as vb
from viss_optimize_ws_b200._lib import DeviceBuffer, check

F32 = np.float32


def dev(a) -> DeviceBuffer:
    return DeviceBuffer.from_array(np.ascontiguousarray(a))


def zeros(n: int, dtype=F32) -> DeviceBuffer:
    b = DeviceBuffer(int(n) * np.dtype(dtype).itemsize)
    b.zero()
    return b


def get(b: DeviceBuffer, dtype=F32, n=None) -> np.ndarray:
    return b.to_array(dtype, n)


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def vp(b) -> C.c_void_p | None:
    if b is None:
        return None
    return C.c_void_p(b.ptr if isinstance(b, DeviceBuffer) else int(b))


def geometry(nside: int):
    """Device l, m, n (library kernel) and host copies."""
    npix = 12 * nside * nside
    l, m, n = zeros(npix), zeros(npix), zeros(npix)
    check(vb.lib().vb_pix2lmn_nest(nside, 0, npix, l.ptr, m.ptr, n.ptr, None))
    return (l, m, n), (get(l), get(m), get(n))


BL_KEYS = ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2")


def reference_baselines(lam: float, day: int, seed: int, t0: int, tlen: int):
    """Baselines of the upstream lunar formation from the library generator:
    host dict (u..z2, invn1, invn2) and device buffers."""
    op = vb.OrbitParams(model=vb.ORBIT_REFERENCE, lambda_m=lam, day=day, seed=seed, nsat=8)
    h = C.c_void_p()
    check(vb.lib().vb_orbit_create(C.byref(op), C.byref(h)))
    n = 56 * tlen
    d = {k: zeros(n) for k in BL_KEYS}
    check(vb.lib().vb_orbit_make_segment(h, t0, tlen, *[d[k].ptr for k in BL_KEYS], None, None, None))
    vb.lib().vb_orbit_destroy(h)
    d["invn1"], d["invn2"] = zeros(n), zeros(n)
    check(vb.lib().vb_invnorm3(d["x1"].ptr, d["y1"].ptr, d["z1"].ptr, d["invn1"].ptr, n, None))
    check(vb.lib().vb_invnorm3(d["x2"].ptr, d["y2"].ptr, d["z2"].ptr, d["invn2"].ptr, n, None))
    host = {k: get(b) for k, b in d.items()}
    host["nbl"] = 28
    return host, d


def synthetic_baselines(nsat: int, T: int, lam: float, seed: int = 42, dt_s: float = 2.0, spread_km: float = 50.0,
                        occ_R_m: float = 6371e3):
    op = vb.OrbitParams(model=vb.ORBIT_SYNTHETIC, lambda_m=lam, day=1, seed=seed, nsat=nsat, tsteps=T, dt_s=dt_s,
                        alt_min_km=400.0, alt_max_km=600.0, spread_km=spread_km, occ_R_m=occ_R_m)
    h = C.c_void_p()
    check(vb.lib().vb_orbit_create(C.byref(op), C.byref(h)))
    nbl = nsat * (nsat - 1) // 2
    n = 2 * nbl * T
    d = {k: zeros(n) for k in BL_KEYS + ("cosphi1", "cosphi2")}
    check(vb.lib().vb_orbit_make_segment(h, 0, T, *[d[k].ptr for k in BL_KEYS], d["cosphi1"].ptr,
                                         d["cosphi2"].ptr, None))
    vb.lib().vb_orbit_destroy(h)
    d["invn1"], d["invn2"] = zeros(n), zeros(n)
    check(vb.lib().vb_invnorm3(d["x1"].ptr, d["y1"].ptr, d["z1"].ptr, d["invn1"].ptr, n, None))
    check(vb.lib().vb_invnorm3(d["x2"].ptr, d["y2"].ptr, d["z2"].ptr, d["invn2"].ptr, n, None))
    host = {k: get(b) for k, b in d.items()}
    host["nbl"] = nbl
    return host, d


def upstream_cosphi() -> float:
    R, h = F32(1737.1e3), F32(300e3)
    theta = np.arcsin(F32(R / (R + h)), dtype=F32)
    phi = F32(np.pi) - theta
    return float(np.cos(phi, dtype=F32))


def sky_struct(dl, dm, dn, dB, npix, tile=None):
    s = vb.Sky()
    s.npix = npix
    s.B, s.l, s.m, s.n = dB.ptr, dl.ptr, dm.ptr, dn.ptr
    if tile is not None:
        tp, (cx, cy, cz, cA, sA) = tile
        s.tile_pix = tp
        s.cx, s.cy, s.cz, s.cosA, s.sinA = cx.ptr, cy.ptr, cz.ptr, cA.ptr, sA.ptr
    return s


def bl_struct(d: dict, n_full: int, nbl: int, cosphi: float, per_end: bool = False):
    b = vb.Baselines()
    b.n_full, b.nbl = n_full, nbl
    for k in BL_KEYS + ("invn1", "invn2"):
        setattr(b, k, d[k].ptr)
    if per_end:
        b.cosphi1, b.cosphi2 = d["cosphi1"].ptr, d["cosphi2"].ptr
    b.cosphi = cosphi
    return b


def tile_meta(tile_pix: int, dl, dm, dn, npix: int):
    nt = (npix + tile_pix - 1) // tile_pix
    arrs = [zeros(nt) for _ in range(5)]
    check(vb.lib().vb_tile_cone_meta(tile_pix, dl.ptr, dm.ptr, dn.ptr, npix, *[a.ptr for a in arrs], None))
    return arrs


def stage1(sky, bls, *, precision, cull, phase_corrected=1, blockage=1, bpt=0, stage_pix=0, chunk_pix=0,
           exact_tile_pix=0, ctas_per_sm=0, items_per_cta=0, refine_pix=0, want_flags=False):
    """vb_viss_halfsym on a fresh workspace: (V_half, term counters), plus the
    workspace's device error word when want_flags is set."""
    o = vb.Stage1Opts(precision=precision, cull=cull, phase_corrected=phase_corrected, blockage=blockage, bpt=bpt,
                      stage_pix=stage_pix, chunk_pix=chunk_pix, exact_tile_pix=exact_tile_pix,
                      ctas_per_sm=ctas_per_sm, items_per_cta=items_per_cta, refine_pix=refine_pix)
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bls), C.byref(o))
    assert need > 0, vb.lib().vb_last_error()
    ws = DeviceBuffer(need)
    n_half = bls.n_full // 2
    V = zeros(2 * n_half, np.float64)
    cnt = zeros(4, np.uint64)
    check(vb.lib().vb_viss_halfsym(C.byref(sky), C.byref(bls), C.byref(o), ws.ptr, need, V.ptr, cnt.ptr, None))
    check(vb.lib().vb_synchronize())
    if want_flags:
        flags = C.c_uint(0xFFFFFFFF)
        check(vb.lib().vb_workspace_error_flags(ws.ptr, C.byref(flags), None))
        return get(V, np.float64), get(cnt, np.uint64), flags.value
    return get(V, np.float64), get(cnt, np.uint64)


def tile_classes(sky, bls, *, cull, precision=vb.PREC_FP32_FP64PH, exact_tile_pix=0, blockage=1,
                 mask_visible_tiles=0):
    o = vb.Stage1Opts(precision=precision, cull=cull, phase_corrected=1, blockage=blockage,
                      exact_tile_pix=exact_tile_pix, mask_visible_tiles=mask_visible_tiles)
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bls), C.byref(o))
    ws = DeviceBuffer(need)
    nt = C.c_int()
    n_half = bls.n_full // 2
    npix = sky.npix
    tile = sky.tile_pix if cull == vb.CULL_TILECONE else (exact_tile_pix or 1024)
    ntile = (npix + tile - 1) // tile
    cls = zeros(n_half * ntile, np.uint8)
    check(vb.lib().vb_stage1_tile_classes(C.byref(sky), C.byref(bls), C.byref(o), ws.ptr, need, cls.ptr,
                                          C.byref(nt), None))
    check(vb.lib().vb_synchronize())
    assert nt.value == ntile
    return get(cls, np.uint8).reshape(n_half, ntile), tile


def stage2(sky, bls, V_half_dev, seg_t0, seg_tlen, *, mirror=1, blockage=1, occ_mode=2, precision=2, cull=0,
           grid_res=0, bl_max=100e3, lam=30.0, ppt=0):
    """vb_recon_batched on device inputs; returns C, W, per-segment params, counters."""
    nseg = len(seg_t0)
    o = vb.Stage2Opts(mirror=mirror, blockage=blockage, occ_mode=occ_mode, precision=precision, cull=cull,
                      grid_res=grid_res, bl_max=bl_max, lambda_=lam, ppt=ppt)
    need = vb.lib().vb_stage2_workspace_bytes(bls.n_full // 2, nseg, sky.npix, C.byref(o))
    assert need > 0, vb.lib().vb_last_error()
    ws = DeviceBuffer(need)
    t0, tl = dev(np.asarray(seg_t0, np.int32)), dev(np.asarray(seg_tlen, np.int32))
    Cb, Wb = zeros(sky.npix), zeros(sky.npix, np.uint32)
    sp = DeviceBuffer(C.sizeof(vb.SegParams) * nseg)
    cnt = zeros(4, np.uint64)
    check(vb.lib().vb_recon_batched(C.byref(sky), C.byref(bls), V_half_dev.ptr, nseg, t0.ptr, tl.ptr, C.byref(o),
                                    ws.ptr, need, Cb.ptr, Wb.ptr, sp.ptr, cnt.ptr, None))
    check(vb.lib().vb_synchronize())
    arr = (vb.SegParams * nseg)()
    check(vb.lib().vb_memcpy(C.addressof(arr), sp.ptr, C.sizeof(arr), 1))
    params = [{k: getattr(a, k) for k, _ in vb.SegParams._fields_} for a in arr]
    return get(Cb), get(Wb, np.uint32), params, get(cnt, np.uint64)
