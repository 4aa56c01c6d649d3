"""Stage-2 parity: plane fit, grid numbers, uv keys, groups and
representatives bit-exact against the upstream kernels / long-double host
formula, and the reconstruction C (and W) against the FP64 CPU oracle on
every path (mirror / full grid, blockage 0 / 1, occ_mode 0 / 1 / 2 / other).

Upstream: viss_recon_kernel.cuh:295-659, 673-701;
..._vissfast.cuh:730-890, 1014-1286; main_recon_online.cu:370-512.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from gpu_util import (bl_struct, dev, geometry, get, reference_baselines, sky_struct, stage1, stage2,
                      upstream_cosphi, vp, zeros)

pytestmark = pytest.mark.gpu

TOL = 1e-5
LAM = float(np.float32(300.0))      # --btag=1M
BL_MAX = 100e3


def half_to_full(ih, nbl):
    ih = np.asarray(ih)
    return (ih // nbl) * 2 * nbl + ih % nbl


@pytest.fixture(scope="module")
def case(gpu, vb):
    nside = 16
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = geometry(nside)
    B = vb.synthetic_sky(nside, seed=5)
    B = (B.astype(np.float64) * (4 * np.pi / npix)).astype(np.float32)
    dB = dev(B)
    tlen = 96
    host, d = reference_baselines(LAM, 1, 42, 100, tlen)
    n_full = host["u"].size
    cp = upstream_cosphi()
    sky = sky_struct(dl, dm, dn, dB, npix)
    bls = bl_struct(d, n_full, 28, cp)
    V, _ = stage1(sky, bls, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_NONE, phase_corrected=1)
    Vh = V.astype(np.float32)
    seg_t0, seg_tlen = [0, 24, 48, 72], [24, 24, 24, 24]
    bl = dict(host)
    bl["cosphi"] = cp
    return dict(npix=npix, sky=sky, bls=bls, dl=dl, dm=dm, dn=dn, skyh=dict(B=B, l=l, m=m, n=n), host=host, d=d,
                bl=bl, Vh=Vh, dVh=dev(Vh), seg_t0=seg_t0, seg_tlen=seg_tlen, cp=cp, n_full=n_full)


def test_seg_params_match_long_double(case, vb, orc):
    c = case
    Cd, W, params, _ = stage2(c["sky"], c["bls"], c["dVh"], c["seg_t0"], c["seg_tlen"], lam=LAM, bl_max=BL_MAX)
    h = c["host"]
    for s, (t0, tl) in enumerate(zip(c["seg_t0"], c["seg_tlen"])):
        i0, n = 56 * t0, 56 * tl
        fa, fb, den = orc.fa_fb(h["u"][i0:i0 + n], h["v"][i0:i0 + n], h["w"][i0:i0 + n])
        p = params[s]
        assert np.float32(p["fa"]) == np.float32(fa) and np.float32(p["fb"]) == np.float32(fb), (s, p, fa, fb)
        R, half, du = orc.grid_params(fa, fb, BL_MAX, LAM)
        assert (p["RES"], p["half"]) == (R, half) and np.float32(p["du"]) == np.float32(du)
        assert np.float32(p["inv_du"]) == np.float32(np.float32(1.0) / np.float32(du))
        # upstream long-double function gives the same floats
        rfa, rfb, rden = np.zeros(1, np.float32), np.zeros(1, np.float32), np.zeros(1)
        orc.ref_root().ref_fa_fb(h["u"][i0:].ctypes.data, h["v"][i0:].ctypes.data, h["w"][i0:].ctypes.data, n,
                                 rfa.ctypes.data, rfb.ctypes.data, rden.ctypes.data)
        assert rfa[0] == np.float32(fa) and rfb[0] == np.float32(fb)


@pytest.mark.parametrize("mirror", [1, 0])
def test_keys_bit_exact_vs_upstream(case, vb, orc, ref, mirror):
    c = case
    h, d = c["host"], c["d"]
    for t0, tl in zip(c["seg_t0"], c["seg_tlen"]):
        i0, n = 56 * t0, 56 * tl
        fa, fb, _ = orc.fa_fb(h["u"][i0:i0 + n], h["v"][i0:i0 + n], h["w"][i0:i0 + n])
        for grid_res in (0, 65):
            R, half, du = orc.grid_params(fa, fb, BL_MAX, LAM, grid_res)
            inv = float(np.float32(1.0) / np.float32(du))
            nk = n // 2 if mirror else n
            mk, rk = zeros(nk, np.int32), zeros(nk, np.int32)
            du_ = C.c_void_p(d["u"].ptr + 4 * i0)
            dv_ = C.c_void_p(d["v"].ptr + 4 * i0)
            vb.check(vb.lib().vb_build_keys(du_.value, dv_.value, nk, 28, mirror, inv, R, half, mk.ptr, None))
            if mirror:
                assert ref.ref_vf().ref_vf_locg_half(du_, dv_, vp(rk), nk, C.c_float(inv), R, half) == 0
            else:
                assert ref.ref_root().ref_locg_full(du_, dv_, vp(rk), nk, C.c_float(inv), R, half) == 0
            mine, theirs = get(mk, np.int32), get(rk, np.int32)
            assert np.array_equal(mine, theirs), f"{int((mine != theirs).sum())} keys differ"
            ok = orc.keys(np.ascontiguousarray(h["u"][i0:i0 + n]), np.ascontiguousarray(h["v"][i0:i0 + n]), nk, 28,
                          mirror, inv, R, half, variant=0)
            assert np.array_equal(ok, mine)


@pytest.mark.parametrize("mirror", [1, 0])
def test_groups_and_representatives_vs_upstream(case, vb, orc, ref, mirror):
    c = case
    h, d = c["host"], c["d"]
    for t0, tl in zip(c["seg_t0"], c["seg_tlen"]):
        i0, n = 56 * t0, 56 * tl
        fa, fb, _ = orc.fa_fb(h["u"][i0:i0 + n], h["v"][i0:i0 + n], h["w"][i0:i0 + n])
        R, half, du = orc.grid_params(fa, fb, BL_MAX, LAM)
        inv = float(np.float32(1.0) / np.float32(du))
        nk = n // 2 if mirror else n
        keys = orc.keys(np.ascontiguousarray(h["u"][i0:i0 + n]), np.ascontiguousarray(h["v"][i0:i0 + n]), nk, 28,
                        mirror, inv, R, half)
        order, uniq, offs = orc.groups(keys)
        nu = np.zeros(1, np.int32)
        ku, cn, of, ix, rp = (np.zeros(nk + 1, np.int32) for _ in range(5))
        va = np.zeros(2 * nk, np.float32)
        du_ = C.c_void_p(d["u"].ptr + 4 * i0)
        dv_ = C.c_void_p(d["v"].ptr + 4 * i0)
        if mirror:
            vh = C.c_void_p(c["dVh"].ptr + 4 * (i0 // 2 * 2))
            assert ref.ref_vf().ref_vf_groups_half(du_, dv_, vh, nk, C.c_float(du), R, half, 1, 2, nu.ctypes.data,
                                                   ku.ctypes.data, cn.ctypes.data, of.ctypes.data, ix.ctypes.data,
                                                   rp.ctypes.data, va.ctypes.data) == 0
            k = int(nu[0])
            assert k == uniq.size and np.array_equal(ku[:k], uniq)
            assert np.array_equal(cn[:k], np.diff(offs))
            reps = order[offs[:-1] + (np.diff(offs) >> 1)]
            assert np.array_equal(rp[:k], reps)
            # the member layout (occ_mode != 2)
            assert ref.ref_vf().ref_vf_groups_half(du_, dv_, vh, nk, C.c_float(du), R, half, 1, 0, nu.ctypes.data,
                                                   ku.ctypes.data, cn.ctypes.data, of.ctypes.data, ix.ctypes.data,
                                                   rp.ctypes.data, va.ctypes.data) == 0
            assert np.array_equal(of[:k + 1], offs) and np.array_equal(ix[:nk], order)
        else:
            vf = zeros(2 * nk)
            assert ref.ref_root().ref_groups_full(du_, dv_, vp(vf), nk, C.c_float(du), R, half, 1, nu.ctypes.data,
                                                  ku.ctypes.data, of.ctypes.data, ix.ctypes.data, va.ctypes.data) == 0
            k = int(nu[0])
            assert k == uniq.size and np.array_equal(ku[:k], uniq)
            assert np.array_equal(of[:k + 1], offs) and np.array_equal(ix[:nk], order)


PATHS = [(1, 1, 2), (1, 1, 0), (1, 1, 1), (1, 1, 3), (1, 0, 2), (0, 1, 2), (0, 1, 0), (0, 1, 3), (0, 0, 2)]


@pytest.mark.parametrize("mirror,blockage,occ", PATHS)
@pytest.mark.parametrize("prec", ["fp32_fp64phase", "fp32_dsphase", "fp64"])
def test_recon_vs_fp64_oracle(case, vb, orc, mirror, blockage, occ, prec):
    c = case
    pm = {"fp64": vb.PREC_FP64, "fp32_fp64phase": vb.PREC_FP32_FP64PH, "fp32_dsphase": vb.PREC_FP32_DSPH}[prec]
    Cd, W, params, cnt = stage2(c["sky"], c["bls"], c["dVh"], c["seg_t0"], c["seg_tlen"], mirror=mirror,
                                blockage=blockage, occ_mode=occ, precision=pm, lam=LAM, bl_max=BL_MAX)
    Co, Wo, sp = orc.stage2(c["skyh"], c["bl"], c["Vh"], c["seg_t0"], c["seg_tlen"], mirror=mirror,
                            blockage=blockage, occ_mode=occ, bl_max=BL_MAX, lam=LAM, precision=1)
    assert [p["nuniq"] for p in params] == list(sp["nuniq"])
    if blockage:
        assert np.array_equal(W, Wo)
    emax, erms = rel_err(Cd, Co)
    tol = 2e-7 if prec == "fp64" else TOL     # FP64 sums, float32 output C
    assert emax <= tol and erms <= tol, f"max {emax:.3e} rms {erms:.3e}"


@pytest.mark.parametrize("ppt", [1, 2, 4])
def test_recon_exact_block_culling_matches_unculled(case, vb, ppt):
    """Exact pixel-block culling changes which groups take the per-pixel test,
    never which groups are included: W identical to the unculled run at every
    block size (256 * ppt pixels); C equal up to the summation order (proven
    visible groups are summed before the mixed ones)."""
    c = case
    proven = 0
    for pm in (vb.PREC_FP32_FP64PH, vb.PREC_FP32_DSPH, vb.PREC_FP64):
        C0, W0, _, k0 = stage2(c["sky"], c["bls"], c["dVh"], c["seg_t0"], c["seg_tlen"], precision=pm, cull=0,
                               lam=LAM, bl_max=BL_MAX, ppt=ppt)
        C1, W1, _, k1 = stage2(c["sky"], c["bls"], c["dVh"], c["seg_t0"], c["seg_tlen"], precision=pm, cull=2,
                               lam=LAM, bl_max=BL_MAX, ppt=ppt)
        assert np.array_equal(W0, W1)
        emax, erms = rel_err(C1, C0)
        tol = 2e-7 if pm == vb.PREC_FP64 else 2e-6
        assert emax <= tol and erms <= tol, (pm, emax, erms)
        assert int(k1[3]) == int(k0[3]) and int(k1[0] + k1[1] + k1[2]) == int(k1[3])
        proven += int(k1[0]) + int(k1[2]) - int(k0[2])
    if ppt == 1:
        assert proven > 0      # 256-pixel blocks: some groups proven visible or hidden


@pytest.mark.parametrize("ppt", [1, 2, 4])
def test_recon_pixels_per_thread_vs_fp64_oracle(case, vb, orc, ppt):
    c = case
    Cd, W, params, cnt = stage2(c["sky"], c["bls"], c["dVh"], c["seg_t0"], c["seg_tlen"], precision=vb.PREC_FP32_FP64PH,
                                cull=2, lam=LAM, bl_max=BL_MAX, ppt=ppt)
    Co, Wo, sp = orc.stage2(c["skyh"], c["bl"], c["Vh"], c["seg_t0"], c["seg_tlen"], mirror=1, blockage=1,
                            occ_mode=2, bl_max=BL_MAX, lam=LAM, precision=1)
    assert np.array_equal(W, Wo)
    emax, erms = rel_err(Cd, Co)
    assert emax <= TOL and erms <= TOL, f"max {emax:.3e} rms {erms:.3e}"


def test_recon_vs_upstream_rep_kernel(case, vb, orc, ref):
    """Mirror occ_mode=2 C and W against the upstream per-segment kernels
    (FP32 fast-math, so C agrees to FP32 level and W exactly)."""
    c = case
    h, d = c["host"], c["d"]
    npix = c["npix"]
    Cacc = np.zeros(npix, np.float64)
    Wacc = np.zeros(npix, np.int64)
    Cseg, Wseg = zeros(npix), zeros(npix, np.uint32)
    for t0, tl in zip(c["seg_t0"], c["seg_tlen"]):
        i0, n = 56 * t0, 56 * tl
        fa, fb, _ = orc.fa_fb(h["u"][i0:i0 + n], h["v"][i0:i0 + n], h["w"][i0:i0 + n])
        R, half, du = orc.grid_params(fa, fb, BL_MAX, LAM)
        nk = n // 2
        nu = np.zeros(1, np.int32)
        ku, cn, of, ix, rp = (np.zeros(nk + 1, np.int32) for _ in range(5))
        va = np.zeros(2 * nk, np.float32)
        du_ = C.c_void_p(d["u"].ptr + 4 * i0)
        dv_ = C.c_void_p(d["v"].ptr + 4 * i0)
        vh = C.c_void_p(c["dVh"].ptr + 4 * (i0 // 2 * 2))
        assert ref.ref_vf().ref_vf_groups_half(du_, dv_, vh, nk, C.c_float(du), R, half, 1, 2, nu.ctypes.data,
                                               ku.ctypes.data, cn.ctypes.data, of.ctypes.data, ix.ctypes.data,
                                               rp.ctypes.data, va.ctypes.data) == 0
        k = int(nu[0])
        keys = ku[:k]
        U, V = (keys - 1) // R, (keys - 1) % R
        ugu = ((U - half).astype(np.float32) * np.float32(du)).astype(np.float32)
        vgu = ((V - half).astype(np.float32) * np.float32(du)).astype(np.float32)
        xs = {kk: C.c_void_p(d[kk].ptr + 4 * i0) for kk in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2", "invn2")}
        dk, du_g, dv_g, drp = dev(keys), dev(ugu), dev(vgu), dev(rp[:k].copy())   # held alive across the call
        assert ref.ref_vf().ref_vf_recon_rep(C.c_longlong(npix), vp(c["dl"]), vp(c["dm"]), vp(c["dn"]),
                                             vp(dk), vp(du_g), vp(dv_g), vp(drp), k, vh,
                                             *[xs[kk] for kk in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2",
                                                                 "invn2")],
                                             C.c_float(fa), C.c_float(fb), C.c_float(c["cp"]), vp(Cseg),
                                             vp(Wseg)) == 0
        Cacc += get(Cseg)
        Wacc += get(Wseg, np.uint32)
    Cup = np.where(Wacc > 0, Cacc / np.maximum(Wacc, 1), 0.0)
    Cd, W, _, _ = stage2(c["sky"], c["bls"], c["dVh"], c["seg_t0"], c["seg_tlen"], lam=LAM, bl_max=BL_MAX)
    assert np.array_equal(W.astype(np.int64), Wacc)
    emax, erms = rel_err(Cup, Cd)
    assert emax < 2e-3 and erms < 2e-3, (emax, erms)
