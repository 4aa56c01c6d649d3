"""Bit-exact parity of the geometry and orbit kernels with the upstream
kernels themselves (run through oracle/_ref on the same GPU): l, m, n, nm1,
tile cones, tile classification, endpoint norms, online uvw/xyz.

Upstream: viss_recon_kernel.cuh:29-112 (pix2lmn), ..._vissfast.cuh:21-98
(tile cones, nm1, classify), orbit_online.cuh:48-366, 443-449.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_util import (BL_KEYS, bits, dev, geometry, get, reference_baselines, tile_meta, upstream_cosphi,
                      vp, zeros)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 32, 128, 512])
def test_pix2lmn_bit_exact(gpu, ref, vb, nside):
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    rl, rm, rn = zeros(npix), zeros(npix), zeros(npix)
    assert ref.ref_root().ref_pix2lmn(nside, 0, npix, vp(rl), vp(rm), vp(rn)) == 0
    for a, b in ((l, get(rl)), (m, get(rm)), (n, get(rn))):
        assert np.array_equal(bits(a), bits(b))
    # the mirror variant's copy of the kernel agrees as well
    assert ref.ref_vf().ref_vf_pix2lmn(nside, 0, npix, vp(rl), vp(rm), vp(rn)) == 0
    assert np.array_equal(bits(l), bits(get(rl)))


def test_pix2lmn_chunks_and_fp64(gpu, ref, vb, orc):
    nside = 64
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    # a chunk starting mid-sky equals the corresponding slice
    base, cnt = 12345, 5000
    cl, cm, cn = zeros(cnt), zeros(cnt), zeros(cnt)
    vb.check(vb.lib().vb_pix2lmn_nest(nside, base, cnt, cl.ptr, cm.ptr, cn.ptr, None))
    assert np.array_equal(bits(get(cl)), bits(l[base:base + cnt]))
    # close to the FP64 restatement
    L, M, N = orc.nest_lmn_f64(nside)
    assert max(np.abs(l - L).max(), np.abs(m - M).max(), np.abs(n - N).max()) < 4e-6
    # range / argument errors
    with pytest.raises(vb.VbError):
        vb.check(vb.lib().vb_pix2lmn_nest(nside, npix - 10, 11, cl.ptr, cm.ptr, cn.ptr, None))
    with pytest.raises(vb.VbError):
        vb.check(vb.lib().vb_pix2lmn_nest(3, 0, 1, cl.ptr, cm.ptr, cn.ptr, None))


def test_nm1_bit_exact(gpu, ref, vb):
    nside = 32
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    a, b = zeros(npix), zeros(npix)
    vb.check(vb.lib().vb_build_nm1(dn.ptr, a.ptr, npix, None))
    assert ref.ref_vf().ref_vf_nm1(vp(dn), vp(b), C.c_longlong(npix)) == 0
    assert np.array_equal(bits(get(a)), bits(get(b)))


@pytest.mark.parametrize("nside,tile", [(16, 256), (32, 512), (64, 1024), (128, 4096), (256, 16384), (8, 512)])
def test_tile_cone_meta_bit_exact(gpu, ref, vb, nside, tile):
    npix = 12 * nside * nside
    (dl, dm, dn), _ = geometry(nside)
    mine = tile_meta(tile, dl, dm, dn, npix)
    nt = (npix + tile - 1) // tile
    theirs = [zeros(nt) for _ in range(5)]
    assert ref.ref_vf().ref_vf_tile_meta(tile, vp(dl), vp(dm), vp(dn), C.c_longlong(npix),
                                         *[vp(t) for t in theirs]) == 0
    for a, b in zip(mine, theirs):
        assert np.array_equal(bits(get(a)), bits(get(b)))


def test_classify_bit_exact(gpu, ref, vb):
    rng = np.random.default_rng(7)
    n = 1 << 20
    # realistic cones plus dots concentrated around the decision boundaries
    nside = 64
    (dl, dm, dn), _ = geometry(nside)
    cones = [get(a) for a in tile_meta(256, dl, dm, dn, 12 * nside * nside)]
    k = rng.integers(0, cones[3].size, n)
    cosA, sinA = cones[3][k], cones[4][k]
    cp = upstream_cosphi()
    d = rng.uniform(-1.05, 1.05, n).astype(np.float32)
    # boundary: lower = d cosA - sqrt(1-d^2) sinA ~ cosphi  <=> d ~ cos(acos(cp) - acos(cosA))
    a = np.arccos(np.clip(cosA.astype(np.float64), -1, 1))
    b = np.arccos(cp)
    near = np.cos(b - a) + rng.normal(0, 1e-6, n)
    near2 = np.cos(b + a) + rng.normal(0, 1e-6, n)
    sel = rng.integers(0, 3, n)
    d = np.where(sel == 0, d, np.where(sel == 1, near, near2)).astype(np.float32)
    dd, dA, dS = dev(d), dev(cosA), dev(sinA)
    mv, mh, rv, rh = (zeros(n, np.uint8) for _ in range(4))
    vb.check(vb.lib().vb_classify_tile_cone(dd.ptr, dA.ptr, dS.ptr, cp, n, mv.ptr, mh.ptr, None))
    assert ref.ref_vf().ref_vf_classify(vp(dd), vp(dA), vp(dS), C.c_float(cp), n, vp(rv), vp(rh)) == 0
    assert np.array_equal(get(mv, np.uint8), get(rv, np.uint8))
    assert np.array_equal(get(mh, np.uint8), get(rh, np.uint8))


@pytest.mark.parametrize("lam,day,seed,t0,tlen", [
    (300.0, 1, 42, 0, 64), (30.0, 3, 42, 1000, 200), (10.0, 17, 7, 12345, 96), (300.0, 15, 123, 6000, 980),
])
def test_orbit_reference_model_bit_exact(gpu, ref, vb, lam, day, seed, t0, tlen):
    lam = float(np.float32(lam))
    host, d = reference_baselines(lam, day, seed, t0, tlen)
    n = 56 * tlen
    outs = {k: np.zeros(n, np.float32) for k in BL_KEYS}
    plan = np.zeros(3, np.int32)
    assert ref.ref_root().ref_orbit(C.c_float(lam), day, C.c_ulonglong(seed), t0, tlen,
                                    *[outs[k].ctypes.data for k in BL_KEYS], plan.ctypes.data) == 0
    for k in BL_KEYS:
        assert np.array_equal(bits(host[k]), bits(outs[k])), k
    # plan numbers agree with the CPU restatement
    assert tuple(plan) == orc_plan(ref, lam)
    # endpoint norms
    for xs, inv in (("1", "invn1"), ("2", "invn2")):
        r = zeros(n)
        assert ref.ref_root().ref_invnorm3(vp(d["x" + xs]), vp(d["y" + xs]), vp(d["z" + xs]), vp(r), n) == 0
        assert np.array_equal(bits(host[inv]), bits(get(r)))
    # upstream +/- layout check passes on both
    assert ref.ref_root().ref_validate_halfsym(outs["u"].ctypes.data, outs["v"].ctypes.data,
                                               outs["w"].ctypes.data, n) == 1
    bad = C.c_int()
    assert vb.lib().vb_validate_uvw_halfsym(d["u"].ptr, d["v"].ptr, d["w"].ptr, n, 28, C.byref(bad), None) == 0


def orc_plan(orc, lam):
    return orc.reference_plan(lam)


def test_validate_halfsym_detects_corruption(gpu, vb, ref):
    host, d = reference_baselines(30.0, 1, 42, 0, 32)
    n = 56 * 32
    u = host["u"].copy()
    u[56 * 7 + 3] += 1.0                      # step 7, pair 3 of the "-" group
    du = dev(u)
    bad = C.c_int()
    rc = vb.lib().vb_validate_uvw_halfsym(du.ptr, d["v"].ptr, d["w"].ptr, n, 28, C.byref(bad), None)
    assert rc == vb._lib.VB_ERR_HALFSYM and bad.value == 56 * 7 + 3
    assert ref.ref_root().ref_validate_halfsym(u.ctypes.data, host["v"].ctypes.data, host["w"].ctypes.data, n) == 0


def test_orbit_window_and_plan_vs_cpu(gpu, vb, orc):
    for lam in (300.0, 30.0, 10.0):
        lam = float(np.float32(lam))
        op = vb.OrbitParams(model=vb.ORBIT_REFERENCE, lambda_m=lam, day=2, seed=5, nsat=8)
        h = C.c_void_p()
        vb.check(vb.lib().vb_orbit_create(C.byref(op), C.byref(h)))
        T, nbl, orr, pc, sl = (C.c_int() for _ in range(5))
        vb.check(vb.lib().vb_orbit_info(h, C.byref(T), C.byref(nbl), C.byref(orr), C.byref(pc), C.byref(sl)))
        vb.lib().vb_orbit_destroy(h)
        assert (orr.value, pc.value, sl.value) == orc.reference_plan(lam)
        assert T.value == pc.value * sl.value and nbl.value == 28


@pytest.mark.parametrize("first", [2 ** 31 - 32768, 12 * 16384 ** 2 - 65536])
def test_nside16384_pixel_indices_beyond_int32(gpu, ref, vb, orc, first):
    """The upstream's 30 MHz default sky is nside 16384: 3.2e9 pixels, so pixel
    indices pass 2^31 (main_recon_online.cu:33-37).  For 65,536 pixels that
    straddle 2^31 (the end of face 7 and the south-polar start of face 8) and
    for the last 65,536 of the sky, the geometry is bit-identical to the
    upstream kernel's, and stage 1 over those pixels matches the FP64 oracle
    (with exact culling bit-identical to none).

    Against the FP64 restatement the float geometry is within 4e-6, except
    close to a pole: the upstream formula takes sin(theta) from a float z, so
    l and m carry an error of about ulp(z) / sin(theta) there (2e-4 at the
    pixels next to the pole at this nside), which the bound follows."""
    from conftest import rel_err
    from gpu_util import bl_struct, reference_baselines, sky_struct, stage1
    nside, cnt = 16384, 65536
    cl, cm, cn = zeros(cnt), zeros(cnt), zeros(cnt)
    vb.check(vb.lib().vb_pix2lmn_nest(nside, first, cnt, cl.ptr, cm.ptr, cn.ptr, None))
    rl, rm, rn = zeros(cnt), zeros(cnt), zeros(cnt)
    assert ref.ref_root().ref_pix2lmn(nside, first, cnt, vp(rl), vp(rm), vp(rn)) == 0
    l, m, n = get(cl), get(cm), get(cn)
    for a, b in ((l, get(rl)), (m, get(rm)), (n, get(rn))):
        assert np.array_equal(bits(a), bits(b))
    L, M, N = orc.nest_lmn_f64(nside, first, cnt)
    bound = 4e-6 + 4e-7 / np.maximum(np.hypot(L, M), 1e-12)
    assert (np.abs(l - L) <= bound).all() and (np.abs(m - M) <= bound).all()
    assert np.abs(n - N).max() < 4e-6
    B = (np.random.default_rng(11).random(cnt) * 1e-3).astype(np.float32)
    dB = dev(B)                                   # held for as long as the sky refers to it
    sky = sky_struct(cl, cm, cn, dB, cnt)
    host, d = reference_baselines(float(np.float32(300.0)), 1, 42, 2000, 16)
    n_full = host["u"].size
    bl = bl_struct(d, n_full, 28, upstream_cosphi())
    V, c, f = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_NONE, want_flags=True)
    assert f == 0 and int(c[3]) == cnt * (n_full // 2)
    Vo = orc.stage1(dict(B=B, l=l, m=m, n=n), dict(host, cosphi=upstream_cosphi()), phase_corrected=1, precision=1)
    if np.abs(Vo).max() > 0:
        emax, erms = rel_err(V, Vo)
        assert emax <= 1e-5 and erms <= 1e-5, (emax, erms)
    else:                                         # every pixel hidden from every baseline
        assert np.abs(V).max() == 0
    Ve, ce, fe = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_EXACT, exact_tile_pix=1024,
                        stage_pix=1024, want_flags=True)
    assert fe == 0 and np.array_equal(Ve.view(np.uint64), V.view(np.uint64))
