"""The CPU oracle against golden vectors produced by the upstream kernels
themselves (tests/golden/make_golden.py ran oracle/_ref on a B200).  Discrete
items must agree bit for bit; the FP64 sums agree with the upstream FP32
fast-math sums to FP32 level.  No GPU needed."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, rel_err

F32 = np.float32


def half_to_full(ih, nbl):
    ih = np.asarray(ih)
    return (ih // nbl) * 2 * nbl + ih % nbl


def test_geometry_vs_fp64_restatement(orc):
    g = load_golden("ref_geometry")
    for nside in (4, 16):
        L, M, N = orc.nest_lmn_f64(nside)
        for a, b in ((g[f"l{nside}"], L), (g[f"m{nside}"], M), (g[f"n{nside}"], N)):
            assert np.abs(a.astype(np.float64) - b).max() < 4e-6


def test_orbit_plan_and_halfsym(orc):
    g = load_golden("ref_orbit")
    for tag in ("b1M", "b30M"):
        lam = float(F32(g[f"{tag}_args"][0]))
        assert tuple(int(x) for x in g[f"{tag}_plan"]) == orc.reference_plan(lam)
        u, v, w = g[f"{tag}_u"], g[f"{tag}_v"], g[f"{tag}_w"]
        n = u.size
        t = np.arange(n) // 56
        j = np.arange(n) % 56
        neg = j < 28
        i1 = np.where(neg, np.arange(n) + 28, np.arange(n))
        assert np.array_equal(u[neg], -u[i1[neg]]) and np.array_equal(w[neg], -w[i1[neg]])
        del t


def test_masks_bit_exact_vs_upstream(orc):
    g = load_golden("ref_stage1")
    npix = g["l"].size
    nh = g["u"].size // 2
    f = half_to_full(np.arange(nh), 28)
    cp = float(g["cosphi"][0])
    m1 = orc.occlusion_mask(g["l"], g["m"], g["n"], *(np.ascontiguousarray(g[k][f]) for k in ("x1", "y1", "z1",
                                                                                             "invn1")), cp)
    m2 = orc.occlusion_mask(g["l"], g["m"], g["n"], *(np.ascontiguousarray(g[k][f]) for k in ("x2", "y2", "z2",
                                                                                             "invn2")), cp)
    mine = (m1 & m2).astype(np.uint8)
    up = np.unpackbits(g["mask_plain"], axis=1)[:, :npix]
    assert np.array_equal(mine, up), f"{int((mine != up).sum())} mask bits differ"


def tile_classes_from_masks(up_tile, plain, tile=256):
    nh, npix = up_tile.shape
    nt = npix // tile
    a = up_tile.reshape(nh, nt, tile)
    p = plain.reshape(nh, nt, tile)
    cls = np.full((nh, nt), 2, np.uint8)
    cls[(a == 1).all(axis=2) & ~(p == 1).all(axis=2)] = 1
    cls[(a == 0).all(axis=2) & ~(p == 0).all(axis=2)] = 0
    return cls


def test_stage1_vs_upstream_fp32(orc):
    g = load_golden("ref_stage1")
    npix = g["l"].size
    sky = dict(B=g["B"], l=g["l"], m=g["m"], n=g["n"])
    bl = {k: g[k] for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2")}
    bl["nbl"] = 28
    bl["cosphi"] = float(g["cosphi"][0])
    V64 = orc.stage1(sky, bl, phase_corrected=0, precision=1)
    e = rel_err(g["V_plain"].astype(np.float64), V64)
    assert e[0] < 5e-4 and e[1] < 5e-4, e
    V32 = orc.stage1(sky, bl, phase_corrected=0, precision=0)
    e32 = rel_err(g["V_plain"].astype(np.float64), V32)
    assert e32[0] < 5e-4, e32
    # tile-cone semantics: the decoded upstream decisions, applied by the oracle
    up_t = np.unpackbits(g["mask_tile"], axis=1)[:, :npix]
    up_p = np.unpackbits(g["mask_plain"], axis=1)[:, :npix]
    cls = tile_classes_from_masks(up_t, up_p)
    # mixed tiles must use exactly the per-pixel mask
    per = np.repeat(cls, 256, axis=1)
    assert np.array_equal(up_t[per == 2], up_p[per == 2])
    Vt = orc.stage1(sky, bl, phase_corrected=0, tile_pix=256, tile_cls=cls, precision=1)
    et = rel_err(g["V_tile"].astype(np.float64), Vt)
    assert et[0] < 5e-4 and et[1] < 5e-4, et


def test_stage2_discrete_items_vs_upstream(orc):
    g = load_golden("ref_stage2")
    nside, lam, bl_max, cp = g["meta"]
    for s in range(4):
        i0, n = 56 * 16 * s, 56 * 16
        u, v, w = (np.ascontiguousarray(g[k][i0:i0 + n]) for k in ("u", "v", "w"))
        fa, fb, den = orc.fa_fb(u, v, w)
        assert F32(fa) == g[f"s{s}_fa"][0] and F32(fb) == g[f"s{s}_fb"][0]
        assert den == g[f"s{s}_denom"][0]
        R, half, du = orc.grid_params(fa, fb, float(bl_max), float(lam))
        inv = float(F32(1.0) / F32(du))
        kh = orc.keys(u, v, n // 2, 28, 1, inv, R, half, variant=0)
        kf = orc.keys(u, v, n, 28, 0, inv, R, half, variant=0)
        assert np.array_equal(kh, g[f"s{s}_keys_half"]), "half-grid keys"
        assert np.array_equal(kf, g[f"s{s}_keys_full"]), "full-grid keys"
        order, uniq, offs = orc.groups(kh)
        assert np.array_equal(uniq, g[f"s{s}_half_uniq"])
        assert np.array_equal(np.diff(offs), g[f"s{s}_half_counts"])
        assert np.array_equal(order, g[f"s{s}_half_order"]) and np.array_equal(offs, g[f"s{s}_half_offsets"])
        reps = order[offs[:-1] + (np.diff(offs) >> 1)]
        assert np.array_equal(reps, g[f"s{s}_half_rep"])
        of, uf, offf = orc.groups(kf)
        assert np.array_equal(uf, g[f"s{s}_full_uniq"]) and np.array_equal(offf, g[f"s{s}_full_offsets"])
        assert np.array_equal(of, g[f"s{s}_full_order"])


def test_stage2_recon_vs_upstream(orc):
    g = load_golden("ref_stage2")
    nside, lam, bl_max, cp = g["meta"]
    geo = load_golden("ref_stage1")
    sky = dict(l=geo["l"], m=geo["m"], n=geo["n"])
    bl = {k: g[k] for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2")}
    bl["nbl"] = 28
    bl["cosphi"] = float(cp)
    t0, tl = [0, 16, 32, 48], [16] * 4
    for tag, mirror, occ in (("rep", 1, 2), ("full2", 0, 2), ("full0", 0, 0)):
        Co, Wo, _ = orc.stage2(sky, bl, g["V_half"], t0, tl, mirror=mirror, occ_mode=occ, bl_max=float(bl_max),
                               lam=float(lam), precision=1)
        assert np.array_equal(Wo.astype(np.int64), g[f"W_{tag}"]), tag
        e = rel_err(g[f"C_{tag}"], Co)
        assert e[0] < 2e-3 and e[1] < 2e-3, (tag, e)
