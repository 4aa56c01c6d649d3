"""Stage-1 parity: the library's visibility sum against
  - the FP64 CPU oracle (numerics; tolerance 1e-5 normwise for the mixed
    precision modes, per the metric's <= 1e-5 relative error bar),
  - the upstream kernels (bit-exact effective occlusion masks and tile
    decisions, decoded by summing powers of two with u = v = w = 0).

Upstream: viss_partial_all_halfsym (viss_recon_kernel.cuh:200-287),
viss_partial_all_halfsym_tilecone (..._vissfast.cuh:437-561).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from gpu_util import (BL_KEYS, bl_struct, dev, geometry, get, reference_baselines, sky_struct, stage1,
                      synthetic_baselines, tile_classes, tile_meta, upstream_cosphi, vp, zeros)

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-5      # max and RMS normwise relative error vs the FP64 oracle
TOL_FP64 = 1e-11
TOL_REF32 = 2e-2


def scaled_sky(vb, nside, seed=3):
    B = vb.synthetic_sky(nside, seed=seed)
    npix = B.size
    return (B.astype(np.float64) * (4.0 * np.pi / npix)).astype(np.float32)


def half_to_full(ih, nbl):
    ih = np.asarray(ih)
    return (ih // nbl) * 2 * nbl + ih % nbl


@pytest.fixture(scope="module")
def case(gpu, vb):
    nside = 32
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    B = scaled_sky(vb, nside)
    dB = dev(B)
    lam = float(np.float32(300.0))
    host, d = reference_baselines(lam, 1, 42, 2000, 16)
    n_full = host["u"].size
    cp = upstream_cosphi()
    tiles = tile_meta(256, dl, dm, dn, npix)
    return dict(nside=nside, npix=npix, dl=dl, dm=dm, dn=dn, l=l, m=m, n=n, B=B, dB=dB, host=host, d=d,
                n_full=n_full, nbl=28, cosphi=cp, tiles=tiles,
                sky=dict(B=B, l=l, m=m, n=n))


def structs(c, tile=True):
    sky = sky_struct(c["dl"], c["dm"], c["dn"], c["dB"], c["npix"], (256, c["tiles"]) if tile else None)
    bl = bl_struct(c["d"], c["n_full"], c["nbl"], c["cosphi"])
    return sky, bl


def bl_dict(c):
    b = dict(c["host"])
    b["cosphi"] = c["cosphi"]
    return b


def test_mask_fma_order_matches_oracle(case, vb, orc):
    c = case
    h = c["host"]
    idx = np.arange(0, c["n_full"], 7)
    x, y, z, inv = (np.ascontiguousarray(h[k][idx]) for k in ("x1", "y1", "z1", "invn1"))
    ne = idx.size
    mk = zeros(ne * c["npix"], np.uint8)
    dx, dy, dz, di = dev(x), dev(y), dev(z), dev(inv)      # held alive across the call
    vb.check(vb.lib().vb_occlusion_mask(c["dl"].ptr, c["dm"].ptr, c["dn"].ptr, c["npix"], dx.ptr, dy.ptr, dz.ptr,
                                        di.ptr, None, c["cosphi"], ne, mk.ptr, None))
    mine = get(mk, np.uint8).reshape(ne, c["npix"])
    v0 = orc.occlusion_mask(c["l"], c["m"], c["n"], x, y, z, inv, c["cosphi"], variant=0)
    v1 = orc.occlusion_mask(c["l"], c["m"], c["n"], x, y, z, inv, c["cosphi"], variant=1)
    d0, d1 = int((mine != v0).sum()), int((mine != v1).sum())
    assert d0 == 0, f"oracle variant 0 differs in {d0} entries (variant 1: {d1})"


def decode_upstream_masks(c, ref, kernel):
    """Effective inclusion of every (half-baseline, pixel) pair by the upstream
    kernel: u=v=w=0, B_p = 2^k on blocks of 16 pixels -> V.x = sum of included 2^k."""
    npix, nh = c["npix"], c["n_full"] // 2
    zero = zeros(c["n_full"])
    Bblk = dev((2.0 ** np.arange(16)).astype(np.float32))
    out = np.zeros((nh, npix), np.uint8)
    Vp = zeros(2 * nh)
    d = c["d"]
    for p0 in range(0, npix, 16):
        off = 4 * p0
        if kernel == "plain":
            rc = ref.ref_root().ref_viss_halfsym(
                vp(Bblk), C.c_void_p(c["dl"].ptr + off), C.c_void_p(c["dm"].ptr + off), C.c_void_p(c["dn"].ptr + off),
                C.c_longlong(16), vp(zero), vp(zero), vp(zero), vp(d["x1"]), vp(d["y1"]), vp(d["z1"]),
                vp(d["invn1"]), vp(d["x2"]), vp(d["y2"]), vp(d["z2"]), vp(d["invn2"]), nh, C.c_float(c["cosphi"]),
                vp(Vp))
        else:
            t = p0 // 256
            toff = 4 * t
            nm1 = zeros(16)
            rc = ref.ref_vf().ref_vf_viss_tilecone(
                256, vp(Bblk), C.c_void_p(c["dl"].ptr + off), C.c_void_p(c["dm"].ptr + off),
                C.c_void_p(c["dn"].ptr + off), vp(nm1), C.c_longlong(16),
                *[C.c_void_p(a.ptr + toff) for a in c["tiles"]], 1, vp(zero), vp(zero), vp(zero), vp(d["x1"]),
                vp(d["y1"]), vp(d["z1"]), vp(d["invn1"]), vp(d["x2"]), vp(d["y2"]), vp(d["z2"]), vp(d["invn2"]), nh,
                C.c_float(c["cosphi"]), vp(Vp))
        assert rc == 0
        vx = get(Vp)[0::2].astype(np.int64)
        for k in range(16):
            out[:, p0 + k] = (vx >> k) & 1
    return out


def my_effective_masks(c, orc, cls=None, tile=256):
    h = c["host"]
    nh = c["n_full"] // 2
    f = half_to_full(np.arange(nh), c["nbl"])
    m1 = orc.occlusion_mask(c["l"], c["m"], c["n"], *(np.ascontiguousarray(h[k][f]) for k in ("x1", "y1", "z1", "invn1")),
                            c["cosphi"])
    m2 = orc.occlusion_mask(c["l"], c["m"], c["n"], *(np.ascontiguousarray(h[k][f]) for k in ("x2", "y2", "z2", "invn2")),
                            c["cosphi"])
    eff = (m1 & m2).astype(np.uint8)
    if cls is not None:
        per_pix = np.repeat(cls, tile, axis=1)[:, :c["npix"]]
        eff = np.where(per_pix == 1, 1, np.where(per_pix == 0, 0, eff)).astype(np.uint8)
    return eff


def test_effective_masks_match_upstream_plain(case, ref, orc):
    up = decode_upstream_masks(case, ref, "plain")
    mine = my_effective_masks(case, orc)
    assert np.array_equal(up, mine), f"{int((up != mine).sum())} differing (baseline, pixel) decisions"


def test_tile_classes_and_masks_match_upstream_tilecone(case, vb, ref, orc):
    sky, bl = structs(case)
    cls, tile = tile_classes(sky, bl, cull=vb.CULL_TILECONE)
    up = decode_upstream_masks(case, ref, "tilecone")
    mine = my_effective_masks(case, orc, cls, tile)
    assert np.array_equal(up, mine), f"{int((up != mine).sum())} differing (baseline, pixel) decisions"
    # all three classes occur in this case (the test exercises every path)
    assert set(np.unique(cls)) == {0, 1, 2}


@pytest.mark.parametrize("cull", ["none", "tilecone", "exact"])
@pytest.mark.parametrize("prec", ["fp64", "fp32_fp64phase", "fp32_dsphase", "ref32"])
def test_stage1_vs_fp64_oracle(case, vb, orc, cull, prec):
    c = case
    sky, bl = structs(c)
    cm = {"none": vb.CULL_NONE, "tilecone": vb.CULL_TILECONE, "exact": vb.CULL_EXACT}[cull]
    pm = {"fp64": vb.PREC_FP64, "fp32_fp64phase": vb.PREC_FP32_FP64PH, "fp32_dsphase": vb.PREC_FP32_DSPH,
          "ref32": vb.PREC_REF32}[prec]
    for pc in (1, 0):
        V, cnt = stage1(sky, bl, precision=pm, cull=cm, phase_corrected=pc)
        cls = None
        if cm == vb.CULL_TILECONE:
            cls, _ = tile_classes(sky, bl, cull=cm)
        Vo = orc.stage1(c["sky"], bl_dict(c), phase_corrected=pc, tile_pix=256 if cls is not None else 0,
                        tile_cls=cls, precision=1)
        emax, erms = rel_err(V, Vo)
        tol = {"fp64": TOL_FP64, "ref32": TOL_REF32}.get(prec, TOL_MIXED)
        assert emax <= tol and erms <= tol, f"{prec}/{cull}/pc={pc}: max {emax:.3e} rms {erms:.3e}"
        assert int(cnt[3]) == c["npix"] * (c["n_full"] // 2)
        assert int(cnt[0] + cnt[1] + cnt[2]) == int(cnt[3])


@pytest.mark.parametrize("prec", ["fp64", "fp32_fp64phase", "fp32_dsphase"])
def test_exact_culling_is_bit_identical_to_per_pixel_masks(case, vb, prec):
    sky, bl = structs(case)
    pm = {"fp64": vb.PREC_FP64, "fp32_fp64phase": vb.PREC_FP32_FP64PH, "fp32_dsphase": vb.PREC_FP32_DSPH}[prec]
    V0, c0 = stage1(sky, bl, precision=pm, cull=vb.CULL_NONE, exact_tile_pix=1024, stage_pix=1024)
    for et in (256, 1024):
        V1, c1 = stage1(sky, bl, precision=pm, cull=vb.CULL_EXACT, exact_tile_pix=et, stage_pix=min(et, 1024))
        if et == 1024:
            assert np.array_equal(V0.view(np.uint64), V1.view(np.uint64))
        else:
            assert rel_err(V1, V0)[0] < 1e-6
        assert int(c1[2]) > 0          # some tiles proven hidden
        assert int(c1[0]) > 0          # some tiles proven visible


def test_stage1_close_to_upstream_fp32(case, vb, ref):
    c = case
    sky, bl = structs(c)
    nh = c["n_full"] // 2
    d = c["d"]
    Vp = zeros(2 * nh)
    assert ref.ref_root().ref_viss_halfsym(vp(c["dB"]), vp(c["dl"]), vp(c["dm"]), vp(c["dn"]),
                                           C.c_longlong(c["npix"]), *[vp(d[k]) for k in ("u", "v", "w")],
                                           *[vp(d[k]) for k in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2",
                                                                "invn2")], nh, C.c_float(c["cosphi"]), vp(Vp)) == 0
    V, _ = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_NONE, phase_corrected=0)
    emax, erms = rel_err(get(Vp).astype(np.float64), V)
    assert emax < 1e-3 and erms < 1e-3, (emax, erms)


def test_stage1_configs_and_determinism(case, vb):
    sky, bl = structs(case)
    Va, _ = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE)
    Vb, _ = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE)
    assert np.array_equal(Va.view(np.uint64), Vb.view(np.uint64))
    for bpt, stg, ch in ((1, 256, 256), (2, 128, 512), (4, 256, 1024)):
        Vc, _ = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, bpt=bpt, stage_pix=stg,
                       chunk_pix=ch)
        assert rel_err(Vc, Va)[0] < 2e-6


@pytest.mark.parametrize("bpt,ctas,items", [(1, 3, 12), (2, 3, 48), (2, 2, 6), (4, 2, 24), (1, 2, 96)])
@pytest.mark.parametrize("prec", ["fp32_fp64phase", "fp64"])
def test_kernel_shapes_vs_fp64_oracle(case, vb, orc, bpt, ctas, items, prec):
    """Every kernel shape the autotuner may pick (baselines per thread,
    resident CTAs per SM, work granularity) gives the oracle's V, the same
    term counters, and per-shape deterministic bits."""
    c = case
    sky, bl = structs(c)
    pm = vb.PREC_FP64 if prec == "fp64" else vb.PREC_FP32_FP64PH
    V, cnt = stage1(sky, bl, precision=pm, cull=vb.CULL_TILECONE, bpt=bpt, ctas_per_sm=ctas, items_per_cta=items)
    V2, cnt2 = stage1(sky, bl, precision=pm, cull=vb.CULL_TILECONE, bpt=bpt, ctas_per_sm=ctas, items_per_cta=items)
    assert np.array_equal(V.view(np.uint64), V2.view(np.uint64))
    cls, _ = tile_classes(sky, bl, cull=vb.CULL_TILECONE)
    Vo = orc.stage1(c["sky"], bl_dict(c), phase_corrected=1, tile_pix=256, tile_cls=cls, precision=1)
    emax, erms = rel_err(V, Vo)
    tol = TOL_FP64 if prec == "fp64" else TOL_MIXED
    assert emax <= tol and erms <= tol, f"max {emax:.3e} rms {erms:.3e}"
    # hidden and total terms are shape-independent; the visible / masked split
    # is per warp (a warp takes the masked path when any of its baselines is mixed)
    _, cnt0 = stage1(sky, bl, precision=pm, cull=vb.CULL_TILECONE)
    assert cnt[2] == cnt0[2] and cnt[3] == cnt0[3] and cnt[0] + cnt[1] == cnt0[0] + cnt0[1]


def test_kernel_shape_rejections(case, vb):
    sky, bl = structs(case)
    for kw in (dict(bpt=4, ctas_per_sm=3), dict(ctas_per_sm=5), dict(items_per_cta=-1), dict(bpt=3)):
        o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1, **kw)
        assert vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o)) == 0, kw


def test_phase_correct_expand(case, vb, orc, ref):
    c = case
    nh = c["n_full"] // 2
    sky, bl = structs(c)
    Vraw, _ = stage1(sky, bl, precision=vb.PREC_FP64, cull=vb.CULL_NONE, phase_corrected=0)
    Vcor, _ = stage1(sky, bl, precision=vb.PREC_FP64, cull=vb.CULL_NONE, phase_corrected=1)
    dV = dev(Vraw)
    vh, vf = zeros(2 * nh), zeros(4 * nh)
    vb.check(vb.lib().vb_phase_correct_expand(dV.ptr, c["d"]["w"].ptr, nh, c["nbl"], 0, vh.ptr, vf.ptr, None))
    Vh, Vf = get(vh), get(vf)
    Oh, Of = orc.phase_correct_expand(Vraw, c["host"]["w"], c["nbl"])
    assert rel_err(Vh, Oh)[0] < 1e-7 and rel_err(Vf, Of)[0] < 1e-7
    # correcting the raw sum equals summing the corrected phase directly
    assert rel_err(Vh, Vcor)[0] < 1e-7
    # conjugate completion: V(-b) = conj V(b)
    f = half_to_full(np.arange(nh), c["nbl"])
    assert np.array_equal(Vf[2 * f], Vf[2 * (f + c["nbl"])])
    assert np.array_equal(Vf[2 * f + 1], -Vf[2 * (f + c["nbl"]) + 1])
    # upstream host correction (FP32 cos/sin of a large angle) agrees loosely
    rh, rf = np.zeros(2 * nh, np.float32), np.zeros(4 * nh, np.float32)
    v32 = Vraw.astype(np.float32)                            # held alive across the call
    ref.ref_root().ref_phase_correct_expand(v32.ctypes.data, c["host"]["w"].ctypes.data, nh, rh.ctypes.data,
                                            rf.ctypes.data)
    assert rel_err(rh, Oh)[0] < 1e-3


def test_stage1_synthetic_per_endpoint_horizon(gpu, vb, orc):
    nside = 16
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    B = scaled_sky(vb, nside, seed=11)
    dB = dev(B)
    lam = float(np.float32(30.0))
    host, d = synthetic_baselines(8, 24, lam)
    n_full = host["u"].size
    sky = sky_struct(dl, dm, dn, dB, npix)
    bl = bl_struct(d, n_full, 28, 0.0, per_end=True)
    blh = dict(host)
    blh["cosphi"] = 0.0
    for prec, tol in ((vb.PREC_FP32_FP64PH, TOL_MIXED), (vb.PREC_FP32_DSPH, TOL_MIXED), (vb.PREC_FP64, TOL_FP64)):
        for cull in (vb.CULL_NONE, vb.CULL_EXACT):
            V, _ = stage1(sky, bl, precision=prec, cull=cull)
            Vo = orc.stage1(dict(B=B, l=l, m=m, n=n), blh, precision=1)
            emax, erms = rel_err(V, Vo)
            assert emax <= tol and erms <= tol, (prec, cull, emax, erms)


def test_point_source_analytic(gpu, vb):
    """One unit pixel, no occlusion: V_k = exp(-2 pi i (u l + v m + w n)) exactly in FP64."""
    nside = 8
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    p = 301
    B = np.zeros(npix, np.float32)
    B[p] = 1.0
    dB = dev(B)
    host, d = reference_baselines(float(np.float32(10.0)), 2, 9, 5000, 8)
    bl = bl_struct(d, host["u"].size, 28, upstream_cosphi())
    sky = sky_struct(dl, dm, dn, dB, npix)
    nh = host["u"].size // 2
    f = half_to_full(np.arange(nh), 28)
    t = (host["u"][f].astype(np.float64) * l[p] + host["v"][f].astype(np.float64) * m[p]
         + host["w"][f].astype(np.float64) * n[p])
    ex = np.exp(-2j * np.pi * (t - np.rint(t)))
    for prec, tol in ((vb.PREC_FP32_FP64PH, 2e-6), (vb.PREC_FP32_DSPH, 3e-6), (vb.PREC_FP64, 1e-12)):
        V, _ = stage1(sky, bl, precision=prec, cull=vb.CULL_NONE, blockage=0)
        z = V[0::2] + 1j * V[1::2]
        assert np.abs(z - ex).max() < tol, (prec, np.abs(z - ex).max())


def decode_my_masks(c, vb, cull):
    """Effective inclusion decided by the library's own stage-1 kernel (FP64
    mode, u=v=w=0, B_p = 2^k on 16-pixel blocks)."""
    npix, nh = c["npix"], c["n_full"] // 2
    zero = zeros(c["n_full"])
    Bblk = dev((2.0 ** np.arange(16)).astype(np.float32))
    out = np.zeros((nh, npix), np.uint8)
    d = c["d"]
    bl = vb.Baselines()
    bl.n_full, bl.nbl, bl.cosphi = c["n_full"], c["nbl"], c["cosphi"]
    bl.u = bl.v = bl.w = zero.ptr
    for k in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2", "invn2"):
        setattr(bl, k, d[k].ptr)
    o = vb.Stage1Opts(precision=vb.PREC_FP64, cull=cull, phase_corrected=1, blockage=1)
    sky = vb.Sky()
    sky.npix = 16
    sky.tile_pix = 256
    sky.B = Bblk.ptr
    sky.l, sky.m, sky.n = c["dl"].ptr, c["dm"].ptr, c["dn"].ptr
    sky.cx, sky.cy, sky.cz, sky.cosA, sky.sinA = (a.ptr for a in c["tiles"])
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o))
    ws = zeros(need, np.uint8)
    V = zeros(2 * nh, np.float64)
    for p0 in range(0, npix, 16):
        off = 4 * p0
        sky.l, sky.m, sky.n = c["dl"].ptr + off, c["dm"].ptr + off, c["dn"].ptr + off
        t = p0 // 256
        sky.cx, sky.cy, sky.cz, sky.cosA, sky.sinA = (a.ptr + 4 * t for a in c["tiles"])
        vb.check(vb.lib().vb_viss_halfsym(C.byref(sky), C.byref(bl), C.byref(o), ws.ptr, need, V.ptr, None, None))
        vx = get(V, np.float64)[0::2].astype(np.int64)
        for k in range(16):
            out[:, p0 + k] = (vx >> k) & 1
    return out


@pytest.mark.parametrize("cull", ["none", "tilecone"])
def test_library_kernel_masks_match_upstream(case, vb, ref, cull):
    cm = vb.CULL_NONE if cull == "none" else vb.CULL_TILECONE
    mine = decode_my_masks(case, vb, cm)
    up = decode_upstream_masks(case, ref, "plain" if cull == "none" else "tilecone")
    assert np.array_equal(mine, up), f"{int((mine != up).sum())} differing (baseline, pixel) decisions"


@pytest.mark.parametrize("prec", ["fp32_fp64phase", "fp64", "fp32_dsphase"])
def test_tilecone_subtile_refinement_is_bit_identical(case, vb, prec):
    """Exact sub-tiles inside tile-cone mixed tiles change only which path a
    warp takes (skip / class select / per-pixel test): V is bit-identical with
    refinement off, and the counters move terms from masked to fast / hidden."""
    sky, bl = structs(case)
    pm = {"fp64": vb.PREC_FP64, "fp32_fp64phase": vb.PREC_FP32_FP64PH, "fp32_dsphase": vb.PREC_FP32_DSPH}[prec]
    Voff, coff = stage1(sky, bl, precision=pm, cull=vb.CULL_TILECONE, refine_pix=-1)
    for r in (0, 32, 64, 128):
        V, c = stage1(sky, bl, precision=pm, cull=vb.CULL_TILECONE, refine_pix=r)
        assert np.array_equal(V.view(np.uint64), Voff.view(np.uint64)), r
        assert c[3] == coff[3] and c[1] <= coff[1] and c[0] >= coff[0] and c[2] >= coff[2]


def test_device_error_word_in_the_workspace(vb, case):
    """The stage-1 error word sits at the start of the caller's workspace and
    is read with vb_workspace_error_flags: clear for in-range inputs, and the
    fp32_fp64phase range bit when a baseline's |u| passes 2^26 wavelengths
    (the exact range reduction needs |u|+|v|+|w| < 2^28 turns)."""
    from gpu_util import DeviceBuffer
    sky, bl = structs(case)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1)
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o))
    ws = DeviceBuffer(need)
    V = zeros(case["n_full"], np.float64)
    flags = C.c_uint(12345)
    vb.check(vb.lib().vb_stage1(C.byref(sky), C.byref(bl), C.byref(o), ws.ptr, need, V.ptr, None))
    vb.check(vb.lib().vb_workspace_error_flags(ws.ptr, C.byref(flags), None))
    assert flags.value == 0
    big = case["host"]["u"].copy()
    big[5] = np.float32(1.0e8)                  # one baseline out of range (finite, no index involved)
    du = dev(big)
    bl.u = du.ptr
    vb.check(vb.lib().vb_stage1(C.byref(sky), C.byref(bl), C.byref(o), ws.ptr, need, V.ptr, None))
    vb.check(vb.lib().vb_workspace_error_flags(ws.ptr, C.byref(flags), None))
    assert flags.value == 8                     # VB_DEVERR_PHASE_RANGE
    bl.u = case["d"]["u"].ptr                    # the word is cleared by the next call
    vb.check(vb.lib().vb_stage1(C.byref(sky), C.byref(bl), C.byref(o), ws.ptr, need, V.ptr, None))
    vb.check(vb.lib().vb_workspace_error_flags(ws.ptr, C.byref(flags), None))
    assert flags.value == 0


@pytest.mark.parametrize("prec", ["fp32_fp64phase", "fp64"])
def test_stage1_on_a_shuffled_pixel_order(case, vb, orc, prec):
    """The C-ABI stage 1 takes any pixel arrays, not only HEALPix NEST order:
    the same pixels in a shuffled order (cull tiles then hold scattered
    pixels) match the FP64 oracle on the shuffled arrays, and the term
    counters are those of the ordered sky."""
    c = case
    rng = np.random.default_rng(5)
    perm = rng.permutation(c["npix"])
    sh = {k: np.ascontiguousarray(c["sky"][k][perm]) for k in ("B", "l", "m", "n")}
    dl, dm, dn, dB = (dev(sh[k]) for k in ("l", "m", "n", "B"))
    sky = sky_struct(dl, dm, dn, dB, c["npix"])
    bl = bl_struct(c["d"], c["n_full"], c["nbl"], c["cosphi"])
    pm = {"fp64": vb.PREC_FP64, "fp32_fp64phase": vb.PREC_FP32_FP64PH}[prec]
    V, cnt = stage1(sky, bl, precision=pm, cull=vb.CULL_NONE)
    Vo = orc.stage1(sh, bl_dict(c), phase_corrected=1, precision=1)
    emax, erms = rel_err(V, Vo)
    tol = TOL_FP64 if prec == "fp64" else TOL_MIXED
    assert emax <= tol and erms <= tol, (emax, erms)
    sky0, _ = structs(c, tile=False)
    V0, cnt0 = stage1(sky0, bl, precision=pm, cull=vb.CULL_NONE)
    assert np.array_equal(cnt, cnt0)



@pytest.mark.parametrize("prec", ["fp32_fp64phase", "fp64", "fp32_dsphase"])
@pytest.mark.parametrize("cull", ["none", "tilecone", "exact"])
def test_staging_across_tiles_and_culled_tiles(case, vb, prec, cull):
    """The pixel records reach shared memory by double-buffered bulk copies
    (each tile's first stage fetched after the tile's barrier, the next one
    while the current one is computed; tiles culled for the whole CTA fetch
    nothing).  Chunks of one tile, of eight tiles and of the automatic size
    give the same V up to the grouping of the FP64 chunk sums, the same term
    counters and a clear device error word, with one, two and eight stages
    per tile."""
    sky, bl = structs(case)
    pm = {"fp64": vb.PREC_FP64, "fp32_fp64phase": vb.PREC_FP32_FP64PH, "fp32_dsphase": vb.PREC_FP32_DSPH}[prec]
    cm = {"none": vb.CULL_NONE, "tilecone": vb.CULL_TILECONE, "exact": vb.CULL_EXACT}[cull]
    # 2048: the largest stage, two 96 KB buffers, one CTA per SM
    stages = (128, 1024, 2048) if cull == "none" else (32, 128, 256)
    extra = dict(exact_tile_pix=256) if cull == "exact" else {}
    for st in stages:
        tile = st if cull == "none" else 256
        V0, c0, f0 = stage1(sky, bl, precision=pm, cull=cm, stage_pix=st, chunk_pix=tile, want_flags=True, **extra)
        assert f0 == 0
        if cull != "none":
            assert int(c0[2]) > 0, "no culled tile: the skip path would not run"
        for ch in (8 * tile, 0):
            V1, c1, f1 = stage1(sky, bl, precision=pm, cull=cm, stage_pix=st, chunk_pix=ch, want_flags=True, **extra)
            assert f1 == 0, (st, ch, f1)
            assert np.array_equal(c1, c0), (st, ch)
            emax, _ = rel_err(V1, V0)
            assert emax < 2e-6, (st, ch, emax)


@pytest.mark.parametrize("drop", [1, 77, 1000])
def test_stage1_on_a_ragged_pixel_count(case, vb, orc, drop):
    """A sky whose pixel count is no multiple of the stage (the last stage of
    the last chunk is short, and so is its bulk copy) gives the FP64 oracle's
    V, and exact culling on 1024-pixel tiles gives the unculled V bit for bit."""
    c = case
    npix = c["npix"] - drop
    sh = {k: np.ascontiguousarray(c["sky"][k][:npix]) for k in ("B", "l", "m", "n")}
    dl, dm, dn, dB = (dev(sh[k]) for k in ("l", "m", "n", "B"))
    sky = sky_struct(dl, dm, dn, dB, npix)
    bl = bl_struct(c["d"], c["n_full"], c["nbl"], c["cosphi"])
    Vo = orc.stage1(sh, bl_dict(c), phase_corrected=1, precision=1)
    for st in (128, 1024):
        V, cnt, f = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_NONE, stage_pix=st, want_flags=True)
        assert f == 0 and int(cnt[3]) == npix * (c["n_full"] // 2)
        emax, erms = rel_err(V, Vo)
        assert emax <= TOL_MIXED and erms <= TOL_MIXED, (st, emax, erms)
    Ve, ce, fe = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_EXACT, exact_tile_pix=1024,
                        stage_pix=1024, want_flags=True)
    assert fe == 0 and int(ce[2]) > 0
    assert np.array_equal(Ve.view(np.uint64), V.view(np.uint64))


def test_workspace_alignment_is_checked(case, vb):
    """A workspace that does not start on a 256-byte boundary is refused on
    the host before anything is launched (the pixel records are bulk-copied
    from it, which needs 16-byte aligned addresses)."""
    from gpu_util import DeviceBuffer
    sky, bl = structs(case)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1)
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o))
    ws = DeviceBuffer(need + 256)
    V = zeros(case["n_full"], np.float64)
    rc = vb.lib().vb_viss_halfsym(C.byref(sky), C.byref(bl), C.byref(o), C.c_void_p(ws.ptr + 16), need, V.ptr,
                                  None, None)
    assert rc == 1 and b"aligned" in vb.lib().vb_last_error()


def test_tile_classes_refuse_a_host_buffer(case, vb):
    """vb_stage1_tile_classes writes its output with a kernel: a host buffer
    is refused on the host, before anything is launched."""
    from gpu_util import DeviceBuffer
    sky, bl = structs(case)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1)
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o))
    ws = DeviceBuffer(need)
    host = np.zeros((case["n_full"] // 2) * (case["npix"] // 256), dtype=np.uint8)
    nt = C.c_int()
    rc = vb.lib().vb_stage1_tile_classes(C.byref(sky), C.byref(bl), C.byref(o), ws.ptr, need, host.ctypes.data,
                                         C.byref(nt), None)
    assert rc == 1 and b"device memory" in vb.lib().vb_last_error()
    assert not host.any()
