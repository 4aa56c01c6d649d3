"""CPU tests of the oracle itself: size-independent properties of the
upstream algorithm (no GPU).  The oracle is additionally pinned against
outputs of the upstream kernels in test_oracle_golden.py."""
from __future__ import annotations

import numpy as np
import pytest

F32 = np.float32


def half_to_full(ih, nbl):
    ih = np.asarray(ih)
    return (ih // nbl) * 2 * nbl + ih % nbl


@pytest.fixture(scope="module")
def small(orc):
    nside = 8
    l64, m64, n64 = orc.nest_lmn_f64(nside)
    sky = dict(l=l64.astype(F32), m=m64.astype(F32), n=n64.astype(F32))
    npix = sky["l"].size
    B = orc.make_sky(nside, 3)
    sky["B"] = (B.astype(np.float64) * (4 * np.pi / npix)).astype(F32)
    bl = orc.syn_baselines(6, 12, lam=30.0)
    bl["cosphi"] = float(-np.sqrt(1 - (6371.0 / 6871.0) ** 2))
    return sky, bl


def test_nest_integer_parts(orc):
    for nside in (1, 2, 8, 64):
        face, ix, iy, jr, nr, ks, jp = orc.nest_ints(nside)
        npix = 12 * nside * nside
        # every (face, ix, iy) appears once; ring index / position in range
        key = face.astype(np.int64) * nside * nside + ix.astype(np.int64) * nside + iy
        assert np.unique(key).size == npix
        assert jr.min() >= 1 and jr.max() <= 4 * nside - 1
        assert (jp >= 1).all() and (jp <= 4 * nside).all()
        # ring sizes: 4*nr pixels on ring jr in the polar caps, 4*nside in the belt
        for r in np.unique(jr):
            cnt = int((jr == r).sum())
            assert cnt == 4 * int(nr[jr == r][0])


def test_lmn_unit_and_equal_area(orc):
    nside = 32
    l, m, n = orc.nest_lmn_f64(nside)
    assert np.allclose(l * l + m * m + n * n, 1.0, atol=1e-14)
    # HEALPix rings: z of pixel centres in the equatorial belt are 2/(3 nside) apart
    z = np.unique(np.round(n, 12))
    assert z.size == 4 * nside - 1
    # equal area: mean of n over the sphere ~ 0
    assert abs(n.mean()) < 1e-12


def test_stage1_point_source_and_linearity(orc, small):
    sky, bl = small
    npix = sky["l"].size
    p = 123
    one = dict(sky, B=np.zeros(npix, F32))
    one["B"][p] = 1.0
    V = orc.stage1(one, bl, blockage=0, precision=1)
    nh = V.size // 2
    f = half_to_full(np.arange(nh), bl["nbl"])
    t = (bl["u"][f].astype(np.float64) * sky["l"][p] + bl["v"][f].astype(np.float64) * sky["m"][p]
         + bl["w"][f].astype(np.float64) * sky["n"][p])
    z = V[0::2] + 1j * V[1::2]
    assert np.abs(z - np.exp(-2j * np.pi * (t - np.rint(t)))).max() < 1e-13
    # linearity in B
    V1 = orc.stage1(sky, bl, precision=1)
    two = dict(sky, B=(2 * sky["B"]).astype(F32))
    V2 = orc.stage1(two, bl, precision=1)
    assert np.abs(V2 - 2 * V1).max() <= 1e-12 * np.abs(V1).max()
    # zero baseline: u = v = w = 0 gives the visible flux
    zb = dict(bl, u=np.zeros_like(bl["u"]), v=np.zeros_like(bl["v"]), w=np.zeros_like(bl["w"]))
    V0 = orc.stage1(sky, zb, precision=1)
    assert np.abs(V0[1::2]).max() < 1e-12
    assert (V0[0::2] <= sky["B"].astype(np.float64).sum() + 1e-9).all()


def test_stage1_phase_correction_identity(orc, small):
    sky, bl = small
    Vraw = orc.stage1(sky, bl, phase_corrected=0, precision=1)
    Vcor = orc.stage1(sky, bl, phase_corrected=1, precision=1)
    Vh, Vf = orc.phase_correct_expand(Vraw, bl["w"], bl["nbl"])
    assert np.abs(Vh - Vcor).max() < 1e-11 * np.abs(Vcor).max()
    nh = Vh.size // 2
    f = half_to_full(np.arange(nh), bl["nbl"])
    assert np.array_equal(Vf[2 * f], Vf[2 * (f + bl["nbl"])])
    assert np.array_equal(Vf[2 * f + 1], -Vf[2 * (f + bl["nbl"]) + 1])


def test_stage1_fp32_flavour_close(orc, small):
    sky, bl = small
    V64 = orc.stage1(sky, bl, precision=1)
    V32 = orc.stage1(sky, bl, precision=0)
    e = np.abs(V32 - V64).max() / np.abs(V64).max()
    assert 1e-9 < e < 1e-2


def test_masks_variants_and_tile_semantics(orc, small):
    sky, bl = small
    x, y, z, inv = bl["x1"][:40], bl["y1"][:40], bl["z1"][:40], bl["invn1"][:40]
    m0 = orc.occlusion_mask(sky["l"], sky["m"], sky["n"], x, y, z, inv, bl["cosphi"], 0)
    m1 = orc.occlusion_mask(sky["l"], sky["m"], sky["n"], x, y, z, inv, bl["cosphi"], 1)
    # the two FMA orders disagree only at the rounding level (rare flips at the horizon)
    assert (m0 != m1).mean() < 1e-3
    # tile classes: all-visible (1) / all-hidden (0) override the per-pixel mask
    nh = bl["u"].size // 2
    npix = sky["l"].size
    ntile = npix // 256
    cls = np.full((nh, ntile), 2, np.uint8)
    Vm = orc.stage1(sky, bl, tile_pix=256, tile_cls=cls, precision=1)
    Vn = orc.stage1(sky, bl, precision=1)
    assert np.array_equal(Vm, Vn)
    cls[:] = 0
    assert not orc.stage1(sky, bl, tile_pix=256, tile_cls=cls, precision=1).any()
    cls[:] = 1
    Vall = orc.stage1(sky, bl, tile_pix=256, tile_cls=cls, precision=1)
    Vnob = orc.stage1(sky, bl, blockage=0, precision=1)
    assert np.array_equal(Vall, Vnob)


def test_fa_fb_exact_plane_and_degenerate(orc):
    rng = np.random.default_rng(2)
    u = rng.uniform(-3e3, 3e3, 2000).astype(F32)
    v = rng.uniform(-3e3, 3e3, 2000).astype(F32)
    w = (u.astype(np.float64) * 0.125 - v.astype(np.float64) * 0.375).astype(F32)
    fa, fb, d = orc.fa_fb(u, v, w)
    assert abs(fa - 0.125) < 1e-6 and abs(fb + 0.375) < 1e-6 and d > 0
    # collinear u, v: degenerate denominator is clamped, result finite
    fa, fb, d = orc.fa_fb(u, 2 * u, w)
    assert np.isfinite(fa) and np.isfinite(fb)
    # no data
    fa, fb, d = orc.fa_fb(u[:0], v[:0], w[:0])
    assert fa == 0.0 and fb == 0.0


def test_grid_params_formula(orc):
    lam = float(F32(30.0))
    R, half, du = orc.grid_params(0.0, 0.0, 100e3, lam)
    span = F32(F32(2.0) * F32(100e3)) / F32(lam)
    tr = np.ceil(F32(span * F32(2.0)) * F32(1.0))
    assert R == int(tr + 2 + 1 - np.fmod(tr, 2)) and R % 2 == 1 and half == (R - 1) // 2
    assert np.float32(du) == F32(span / F32(R - 1))
    assert orc.grid_params(0.3, -0.2, 100e3, lam, 512)[0] == 513
    assert orc.grid_params(0.3, -0.2, 100e3, lam, 257)[0] == 257


def test_keys_rounding_rules(orc):
    RES, half = 9, 4
    inv = 1.0
    # full grid: round half away from zero; half grid: floor(x + 0.5)
    u = np.array([0.5, -0.5, 1.49, -1.5, 4.4, 4.6, -4.6], F32)
    v = np.zeros_like(u)
    nbl = u.size
    kf = orc.keys(np.concatenate([u, -u]), np.concatenate([v, v]), nbl, nbl, 0, inv, RES, half, 1)
    Uf = np.where(kf > 0, (kf - 1) // RES - half, -99)
    assert list(Uf) == [1, -1, 1, -2, 4, -99, -99]
    kh = orc.keys(np.concatenate([u, -u]), np.concatenate([v, v]), nbl, nbl, 1, inv, RES, half, 1)
    Uh = np.where(kh > 0, (kh - 1) // RES - half, -99)
    assert list(Uh) == [1, 0, 1, -1, 4, -99, -99]


def test_groups_stable_and_representatives(orc):
    rng = np.random.default_rng(3)
    k = rng.integers(0, 20, 500).astype(np.int32)
    order, uniq, offs = orc.groups(k)
    assert np.array_equal(np.sort(np.unique(k)), uniq)
    assert np.array_equal(k[order], np.sort(k, kind="stable"))
    for q in range(uniq.size):
        members = order[offs[q]:offs[q + 1]]
        assert (np.diff(members) > 0).all()          # index order inside a key
        assert (k[members] == uniq[q]).all()


def test_stage2_paths_consistency(orc, small):
    sky, bl = small
    V = orc.stage1(sky, bl, precision=1)
    Vh = V.astype(F32)
    t0, tl = [0, 6], [6, 6]
    res = {}
    for occ in (0, 1, 2, 3):
        Cc, W, sp = orc.stage2(sky, bl, Vh, t0, tl, mirror=1, occ_mode=occ, grid_res=33, bl_max=100e3, lam=30.0)
        res[occ] = (Cc, W)
        assert np.isfinite(Cc).all() and (W <= sp["nuniq"].sum()).all()
    # a group of one member: occ modes 0, 1, 2, 3 coincide when every group has one member
    Cc0, W0, sp = orc.stage2(sky, bl, Vh, t0, tl, mirror=1, occ_mode=0, grid_res=4001, bl_max=1e6, lam=30.0)
    Cc2, W2, _ = orc.stage2(sky, bl, Vh, t0, tl, mirror=1, occ_mode=2, grid_res=4001, bl_max=1e6, lam=30.0)
    if sp["nuniq"].sum() == Vh.size // 2:
        assert np.allclose(Cc0, Cc2) and np.array_equal(W0, W2)
    # blockage=0 normalises by the total group count
    Cb, Wb, spb = orc.stage2(sky, bl, Vh, t0, tl, mirror=1, blockage=0, grid_res=33, bl_max=100e3, lam=30.0)
    assert not Wb.any() and np.isfinite(Cb).all()


def test_reference_plan_numbers(orc):
    # main_recon_online.cu:116-121 at the three upstream bands
    for lam, orr in ((300.0, 2095), (30.0, 20944), (10.0, 62832)):
        a, b, c = orc.reference_plan(float(F32(lam)))
        assert (a, b, c) == (orr, 10, orr // 3)
    t1 = orc.window_starts(float(F32(300.0)), 3, 42)
    orr, pc, sl = orc.reference_plan(float(F32(300.0)))
    g = np.arange(pc)
    assert (t1 >= g * orr).all() and (t1 + sl - 1 <= (g + 1) * orr - 1).all()


def test_sky_generator_matches_library(orc, vb):
    a = orc.make_sky(8, 11, 20, 10.0)
    b = vb.synthetic_sky(8, seed=11, n_points=20, amp=10.0)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert a.min() >= 0 and (a >= 10).sum() >= 15


def _occ_threshold(invn: np.float32, c: np.float32) -> np.float32:
    """The stage-1 kernel's per-endpoint threshold (occ_threshold), restated in
    numpy float32: the smallest float t with fl(t * invn) >= c."""
    f = np.float32
    if np.isnan(c) or np.isnan(invn):
        return f(-np.inf)
    if invn == 0:
        return f(np.inf) if c > 0 else f(-np.inf)
    if np.isinf(invn):
        return f(0.0)
    t = f(c / invn)
    for _ in range(16):
        if f(t * invn) >= c:
            break
        t = np.nextafter(t, f(np.inf))
    for _ in range(16):
        p = np.nextafter(t, f(-np.inf))
        if f(p * invn) >= c:
            t = p
        else:
            break
    return t


def test_occlusion_threshold_is_exact():
    """The per-pixel occlusion test fl(d * invn) < cosphi is decided in the
    stage-1 kernel as d < t with a per-endpoint float threshold t.  Rounding to
    nearest never decreases as d grows (invn > 0), so the two tests agree for
    every d: checked for random endpoints' invn and horizon cosines, on random
    d and on the 64 floats either side of each threshold, where a slip in t
    would show."""
    rng = np.random.default_rng(17)
    f = np.float32
    for _ in range(400):
        invn = f(1.0 / rng.uniform(1700.0, 45000.0))          # 1 / |endpoint| in km
        c = f(rng.uniform(-1.0, 1.0))
        t = _occ_threshold(invn, c)
        assert f(t * invn) >= c and f(np.nextafter(t, f(-np.inf)) * invn) < c
        d = rng.uniform(-5e4, 5e4, 2000).astype(np.float32)
        near = [t]
        for _ in range(64):
            near.append(np.nextafter(near[-1], f(np.inf)))
        lo = [t]
        for _ in range(64):
            lo.append(np.nextafter(lo[-1], f(-np.inf)))
        d = np.concatenate([d, np.array(near + lo, dtype=np.float32)])
        assert np.array_equal((d * invn).astype(np.float32) < c, d < t)
