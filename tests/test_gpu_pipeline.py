"""Whole-run parity of vb_pipeline (orbit -> stage 1 -> stage 2, one CUDA
graph) against the FP64 CPU oracle on the pipeline's own inputs, plus graph
vs eager, run-to-run determinism and the host-buffer entry point.

Upstream orchestration: main_recon_online.cu:150-512,
main_recon_online_mirror_tile_vissfast.cu:151-604.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from gpu_util import tile_classes

pytestmark = pytest.mark.gpu

TOL = 1e-5


def host_inputs(p):
    keys = ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2", "cosphi1", "cosphi2")
    bl = {k: p.get(k) for k in keys}
    bl = {k: v for k, v in bl.items() if v.size}
    bl["nbl"] = p.nbl
    bl["cosphi"] = p.cosphi
    sky = {k: p.get(k) for k in ("B", "l", "m", "n")}
    return sky, bl


def pipeline_tile_classes(vb, p):
    sky = vb.Sky()
    sky.npix = p.npix
    for k in ("B", "l", "m", "n", "cx", "cy", "cz", "cosA", "sinA"):
        setattr(sky, k, p.ptr(k)[0])
    sky.tile_pix = p.cfg.viss_tile_pix
    bl = vb.Baselines()
    bl.n_full, bl.nbl, bl.cosphi = 2 * p.n_half, p.nbl, p.cosphi
    for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2"):
        setattr(bl, k, p.ptr(k)[0])
    c1, n1 = p.ptr("cosphi1")
    if c1 and n1:                                   # per-endpoint horizon cosines
        bl.cosphi1, bl.cosphi2 = c1, p.ptr("cosphi2")[0]
    cls, tile = tile_classes(sky, bl, cull=vb.CULL_TILECONE, mask_visible_tiles=0 if p.cfg.nm1_fast else 1)
    return cls, tile


@pytest.mark.parametrize("model", ["synthetic", "reference"])
def test_pipeline_vs_oracle(gpu, vb, orc, model):
    if model == "synthetic":
        cfg = vb.run_config(nside=16, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=64, segs=4, lambda_m=30.0,
                            occ_R_m=6371e3, cull="tilecone", viss_tile_pix=256, mirror=1, grid_res=129,
                            bl_max_m=100e3)
    else:
        cfg = vb.run_config(nside=8, orbit_model=vb.ORBIT_REFERENCE, segs=4, lambda_m=vb.btag_lambda("1M"),
                            cull="tilecone", viss_tile_pix=256, mirror=1)
    with vb.Pipeline(cfg) as p:
        B = vb.synthetic_sky(16 if model == "synthetic" else 8, seed=2)
        p.set_sky(B)
        p.make_baselines()
        rep = p.run()
        assert rep["error_flags"] == 0
        Vh = p.get("V_half")
        Cd = p.get("C")
        Wd = p.get("W")
        sky, bl = host_inputs(p)
        cls, tile = pipeline_tile_classes(vb, p)
        Vo = orc.stage1(sky, bl, phase_corrected=1, tile_pix=tile, tile_cls=cls, precision=1)
        emax, erms = rel_err(Vh, Vo)
        assert emax <= TOL and erms <= TOL, (emax, erms)
        t0, tl = p.seg_plan()
        sp = p.seg_params()
        Co, Wo, osp = orc.stage2(sky, bl, Vh, t0, tl, mirror=1, blockage=1, occ_mode=2, bl_max=cfg.bl_max_m,
                                 lam=cfg.lambda_m, grid_res=cfg.grid_res, precision=1)
        assert [s["nuniq"] for s in sp] == list(osp["nuniq"])
        assert [np.float32(s["fa"]) for s in sp] == list(osp["fa"])
        assert np.array_equal(Wd, Wo)
        emax, erms = rel_err(Cd, Co)
        assert emax <= TOL and erms <= TOL, (emax, erms)
        assert rep["stage1_terms"] == p.npix * p.n_half
        assert rep["stage2_terms"] == p.npix * sum(s["nuniq"] for s in sp)


def test_nm1_fast_off_vs_oracle(gpu, vb, orc):
    """--nm1_fast=0: tiles the cone test proves visible take the per-pixel test
    like mixed tiles (upstream's all-visible fast path, ..._vissfast.cuh:530-539,
    switched off); only tiles proven hidden are culled.  Against the oracle
    with the same tile classes, and against the default where they differ."""
    kw = dict(nside=16, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=64, segs=4, lambda_m=30.0,
              occ_R_m=6371e3, cull="tilecone", viss_tile_pix=256, mirror=1, grid_res=129, bl_max_m=100e3)
    B = vb.synthetic_sky(16, seed=2)
    res = {}
    for fast in (1, 0):
        with vb.Pipeline(vb.run_config(nm1_fast=fast, **kw)) as p:
            p.set_sky(B)
            p.make_baselines()
            rep = p.run()
            assert rep["error_flags"] == 0
            cls, tile = pipeline_tile_classes(vb, p)
            res[fast] = (p.get("V_half"), cls, rep["s1_counters"])
            if not fast:
                sky, bl = host_inputs(p)
                Vo = orc.stage1(sky, bl, phase_corrected=1, tile_pix=tile, tile_cls=cls, precision=1)
                emax, erms = rel_err(res[0][0], Vo)
                assert emax <= TOL and erms <= TOL, (emax, erms)
    assert np.any(res[1][1] == 1) and not np.any(res[0][1] == 1)       # no tile is taken as visible
    assert np.array_equal(res[1][1] == 0, res[0][1] == 0)               # the same tiles are culled
    assert res[0][2][3] == res[1][2][3] and res[0][2][2] >= res[1][2][2]  # same nominal terms, no fewer skipped


def test_one_call_run_and_stage_names(gpu, vb):
    """vb_run (one call: create, upload, baselines, both stages, download,
    free) equals the pipeline's host entry bit for bit and rejects a wrong
    buffer size; vb_stage1 / vb_stage2 equal vb_viss_halfsym /
    vb_recon_batched on the pipeline's own device arrays."""
    from gpu_util import DeviceBuffer, dev, get, zeros
    cfg = vb.run_config(nside=16, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=32, segs=2, lambda_m=30.0,
                        occ_R_m=6371e3, cull="tilecone", viss_tile_pix=256, mirror=1, grid_res=65, bl_max_m=100e3)
    B = vb.synthetic_sky(16, seed=5)
    with vb.Pipeline(cfg) as p:
        C1, V1, _ = p.run_host(B, want_v=True)
        npix, n_half = p.npix, p.n_half
        # the stage entries on the pipeline's arrays (after run_host: sky scaled, baselines made)
        sky = vb.Sky()
        sky.npix = npix
        for k in ("B", "l", "m", "n", "cx", "cy", "cz", "cosA", "sinA"):
            setattr(sky, k, p.ptr(k)[0])
        sky.tile_pix = cfg.viss_tile_pix
        bl = vb.Baselines()
        bl.n_full, bl.nbl, bl.cosphi = 2 * n_half, p.nbl, p.cosphi
        for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2", "cosphi1", "cosphi2"):
            setattr(bl, k, p.ptr(k)[0])
        o1 = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1)
        need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o1))
        ws = DeviceBuffer(need)
        Va, Vb = zeros(2 * n_half, np.float64), zeros(2 * n_half, np.float64)
        vb.check(vb.lib().vb_viss_halfsym(C.byref(sky), C.byref(bl), C.byref(o1), ws.ptr, need, Va.ptr, None, None))
        vb.check(vb.lib().vb_stage1(C.byref(sky), C.byref(bl), C.byref(o1), ws.ptr, need, Vb.ptr, None))
        vb.check(vb.lib().vb_synchronize())
        assert np.array_equal(get(Va, np.float64).view(np.uint64), get(Vb, np.float64).view(np.uint64))
        t0, tl = p.seg_plan()
        o2 = vb.Stage2Opts(mirror=1, blockage=1, occ_mode=2, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_EXACT,
                           grid_res=cfg.grid_res, bl_max=cfg.bl_max_m, lambda_=cfg.lambda_m)
        need2 = vb.lib().vb_stage2_workspace_bytes(n_half, len(t0), npix, C.byref(o2))
        ws2 = DeviceBuffer(need2)
        Vh = dev(V1)
        dt0, dtl = dev(np.asarray(t0, np.int32)), dev(np.asarray(tl, np.int32))
        outs = []
        for name in ("vb_recon_batched", "vb_stage2"):
            Cb, Wb = zeros(npix), zeros(npix, np.uint32)
            args = [C.byref(sky), C.byref(bl), Vh.ptr, len(t0), dt0.ptr, dtl.ptr, C.byref(o2), ws2.ptr, need2,
                    Cb.ptr, Wb.ptr]
            args += [None, None, None] if name == "vb_recon_batched" else [None]
            vb.check(getattr(vb.lib(), name)(*args))
            vb.check(vb.lib().vb_synchronize())
            outs.append((get(Cb), get(Wb, np.uint32)))
        assert np.array_equal(outs[0][0].view(np.uint32), outs[1][0].view(np.uint32))
        assert np.array_equal(outs[0][1], outs[1][1])
    C2 = np.empty(npix, np.float32)
    V2 = np.empty(2 * n_half, np.float32)
    rep = vb.Report()
    vb.check(vb.lib().vb_run(C.byref(cfg), B.ctypes.data, 1, npix, C2.ctypes.data, V2.ctypes.data, C.byref(rep)))
    assert np.array_equal(C1.view(np.uint32), C2.view(np.uint32))
    assert np.array_equal(V1.view(np.uint32), V2.view(np.uint32))
    assert rep.error_flags == 0
    assert vb.lib().vb_run(C.byref(cfg), B.ctypes.data, 1, npix + 1, C2.ctypes.data, None, None) == 1   # VB_ERR_INVALID


def test_graph_eager_determinism_and_host_entry(gpu, vb):
    kw = dict(nside=16, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=48, segs=3, lambda_m=30.0, occ_R_m=6371e3,
              cull="exact", mirror=1, grid_res=101)
    B = vb.synthetic_sky(16, seed=9)
    outs = []
    for use_graph in (1, 0, 1):
        with vb.Pipeline(vb.run_config(use_graph=use_graph, **kw)) as p:
            p.set_sky(B)
            p.make_baselines()
            p.run()
            p.run()
            outs.append((p.get("C"), p.get("V_half"), p.get("W")))
            Ch, Vh, r = p.run_host(B, want_v=True)
            assert np.array_equal(Ch.view(np.uint32), outs[-1][0].view(np.uint32))
            assert np.array_equal(Vh.view(np.uint32), outs[-1][1].view(np.uint32))
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_precision_modes_against_fp64_pipeline(gpu, vb):
    """The mixed-precision builds against the plain FP64 build of the same
    pipeline (same tile classes, groups): <= 1e-5 normwise for V and C."""
    kw = dict(nside=32, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=128, segs=4, lambda_m=30.0,
              occ_R_m=6371e3, cull="tilecone", viss_tile_pix=1024, mirror=1, grid_res=257)
    B = vb.synthetic_sky(32, seed=4)
    res = {}
    for prec in ("fp64", "fp32_fp64phase", "fp32_dsphase", "ref32"):
        with vb.Pipeline(vb.run_config(precision=prec, **kw)) as p:
            p.set_sky(B)
            p.make_baselines()
            p.run()
            res[prec] = (p.get("V_half"), p.get("C"))
    for prec in ("fp32_fp64phase", "fp32_dsphase"):
        for i in (0, 1):
            emax, erms = rel_err(res[prec][i], res["fp64"][i])
            assert emax <= TOL and erms <= TOL, (prec, i, emax, erms)
    # the upstream FP32 arithmetic is measurably worse (documents why the phase needs FP64)
    assert rel_err(res["ref32"][0], res["fp64"][0])[1] > 1e-5


def test_halfsym_violation_is_reported(gpu, vb):
    with vb.Pipeline(vb.run_config(nside=8, orbit_model=vb.ORBIT_SYNTHETIC, nsat=4, tsteps=8, segs=2,
                                   lambda_m=30.0, occ_R_m=6371e3, grid_res=33)) as p:
        p.set_sky(vb.synthetic_sky(8))
        p.make_baselines()
        ptr, n = p.ptr("u")
        uh = np.empty(n, np.float32)
        vb.check(vb.lib().vb_memcpy(uh.ctypes.data, ptr, uh.nbytes, 1))
        uh[5] += 3.0
        vb.check(vb.lib().vb_memcpy(ptr, uh.ctypes.data, uh.nbytes, 0))
        bad = C.c_int()
        vp_, _ = p.ptr("v")
        wp_, _ = p.ptr("w")
        rc = vb.lib().vb_validate_uvw_halfsym(ptr, vp_, wp_, n, p.nbl, C.byref(bad), None)
        assert rc == 6 and bad.value == 5


def test_autotune_keeps_results_and_picks_a_valid_shape(gpu, vb):
    """vb_pipeline_autotune times the kernel shapes on the pipeline's own
    inputs, keeps the fastest, and the tuned run gives the untuned run's
    results (to FP32 summation-order rounding; discrete W identical)."""
    kw = dict(nside=32, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=128, segs=4, lambda_m=30.0,
              occ_R_m=6371e3, cull="tilecone", viss_tile_pix=1024, mirror=1, grid_res=257)
    B = vb.synthetic_sky(32, seed=4)
    with vb.Pipeline(vb.run_config(**kw)) as p:
        p.set_sky(B)
        p.make_baselines()
        p.run()
        C0, V0, W0 = p.get("C"), p.get("V_half"), p.get("W")
        t = p.autotune(reps=1)
        assert t["candidates"] >= 20
        assert t["stage1_bpt"] in (1, 2, 4) and t["stage1_ctas_per_sm"] in (2, 3)
        assert t["stage1_stage_pix"] in (256, 512, 1024) and t["stage2_ppt"] in (1, 2, 4)
        assert 0 < t["stage1_ms"] <= t["stage1_default_ms"] and 0 < t["stage2_ms"] <= t["stage2_default_ms"]
        r = p.run()
        assert r["graph_kernels"] > 0 and r["error_flags"] == 0
        C1, V1, W1 = p.get("C"), p.get("V_half"), p.get("W")
        assert np.array_equal(W0, W1)
        assert rel_err(V1, V0)[0] < 2e-6 and rel_err(C1, C0)[0] < 2e-6
        # a second run of the tuned graph is bit-identical
        p.run()
        assert np.array_equal(p.get("C").view(np.uint32), C1.view(np.uint32))


def test_set_day_matches_a_fresh_pipeline(gpu, vb):
    """vb_pipeline_set_day swaps the day's orbit in a live pipeline (buffers,
    plans and graph kept): results are bit-identical to a pipeline created for
    that day; a day with another step count is refused."""
    kw = dict(nside=16, orbit_model=vb.ORBIT_REFERENCE, segs=2, lambda_m=vb.btag_lambda("1M"), mirror=1,
              cull="tilecone", viss_tile_pix=256, grid_res=0, bl_max_m=0.0)
    B = vb.synthetic_sky(16, seed=5)
    with vb.Pipeline(vb.run_config(day=1, **kw)) as p:
        p.set_sky(B)
        p.make_baselines()
        p.run()
        vb.check(vb.lib().vb_pipeline_set_day(p.h, 2))
        r = p.run()
        assert r["error_flags"] == 0
        C2, V2 = p.get("C"), p.get("V_half")
    with vb.Pipeline(vb.run_config(day=2, **kw)) as q:
        q.set_sky(B)
        q.make_baselines()
        q.run()
        assert np.array_equal(q.get("C").view(np.uint32), C2.view(np.uint32))
        assert np.array_equal(q.get("V_half").view(np.uint32), V2.view(np.uint32))
    # synthetic model: tsteps fixed by the config, so any day keeps the shape
    with vb.Pipeline(vb.run_config(nside=8, orbit_model=vb.ORBIT_SYNTHETIC, nsat=4, tsteps=8, segs=2,
                                   lambda_m=30.0, occ_R_m=6371e3, grid_res=33)) as s:
        s.set_sky(vb.synthetic_sky(8))
        s.make_baselines()
        vb.check(vb.lib().vb_pipeline_set_day(s.h, 7))
        s.run()


def test_device_accumulate(gpu, vb):
    from gpu_util import dev, get, zeros
    rng = np.random.default_rng(2)
    a = rng.standard_normal(5000).astype(np.float32)
    acc = zeros(5000, np.float64)
    da = dev(a)
    for _ in range(3):
        vb.check(vb.lib().vb_accumulate(da.ptr, a.size, acc.ptr, None))
    vb.check(vb.lib().vb_synchronize())
    assert np.array_equal(get(acc, np.float64), 3 * a.astype(np.float64))


@pytest.mark.parametrize("prec,slab", [("fp32_fp64phase", 4096), ("fp64", 5120)])
def test_sky_slab_streaming_matches_resident(gpu, vb, prec, slab):
    """slab_pix streams the sky through the device in slabs (geometry per
    slab, B from host memory, V summed over slabs, C written per slab): the
    results equal the resident run's to summation-order rounding and the term
    counters are identical; 5120 leaves a short last slab."""
    kw = dict(nside=32, orbit_model=vb.ORBIT_SYNTHETIC, nsat=8, tsteps=64, segs=3, lambda_m=30.0, occ_R_m=6371e3,
              cull="tilecone", viss_tile_pix=1024, mirror=1, grid_res=129, bl_max_m=0.0, precision=prec)
    B = vb.synthetic_sky(32, seed=6)
    with vb.Pipeline(vb.run_config(**kw)) as p:
        C0, V0, r0 = p.run_host(B, want_v=True)
    with vb.Pipeline(vb.run_config(slab_pix=slab, **kw)) as q:
        C1, V1, r1 = q.run_host(B, want_v=True)
        C2, V2, r2 = q.run_host(B, want_v=True)
        with pytest.raises(vb.VbError):
            q.run()
        with pytest.raises(vb.VbError):
            q.set_sky(B)
    assert r1["s1_counters"] == r0["s1_counters"] and r1["s2_counters"] == r0["s2_counters"]
    assert r1["bl_max_m"] == r0["bl_max_m"] and r1["error_flags"] == 0
    assert rel_err(V1, V0)[0] < 1e-6 and rel_err(C1, C0)[0] < 1e-6
    assert np.array_equal(C2.view(np.uint32), C1.view(np.uint32))


def test_sky_slab_size_must_hold_whole_tiles(gpu, vb):
    with pytest.raises(vb.VbError):
        vb.Pipeline(vb.run_config(nside=32, orbit_model=vb.ORBIT_SYNTHETIC, nsat=4, tsteps=8, segs=2,
                                  lambda_m=30.0, occ_R_m=6371e3, cull="tilecone", viss_tile_pix=2048,
                                  slab_pix=3072))


def test_nside16384_day_in_sky_slabs(gpu, vb, orc):
    """The upstream's 30 MHz default sky is nside 16384 (3.2e9 pixels,
    main_recon_online.cu:33-37), larger than the device holds with its stage-1
    records.  The pipeline streams it in 12 slabs of 2^28 pixels; the sky is
    one point source at pixel 2,750,722,240 (past 2^31) and 4 satellites give
    96 half-baselines.  V is that one pixel's terms: within 1e-5 of the FP64
    oracle on the one-pixel sky, so |V_k| is B where both endpoints see the
    source and 0 where either does not.  C at the source and its neighbours
    matches the oracle's stage 2 on those pixels with the pipeline's V and
    segments, and the term counters hold npix x N_half (past 2^32).  Visible
    tiles take the per-pixel test here (nm1_fast=0), so the one-pixel oracle
    sees the same masks."""
    from gpu_util import get, zeros
    nside = 16384
    npix = 12 * nside * nside
    src = 2_750_722_240                      # seen by about half of the baselines
    kw = dict(nside=nside, orbit_model=vb.ORBIT_SYNTHETIC, nsat=4, tsteps=16, segs=2,
              lambda_m=vb.btag_lambda("30M"), occ_R_m=6371e3, cull="tilecone", viss_tile_pix=16384, mirror=1,
              grid_res=65, bl_max_m=0.0, nm1_fast=0, slab_pix=1 << 28)
    B = np.zeros(npix, dtype=np.float32)
    B[src] = 1.0
    with vb.Pipeline(vb.run_config(**kw)) as p:
        assert p.npix == npix
        Cout, V, rep = p.run_host(B, scale=False, want_v=True)
        keys = ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2", "cosphi1", "cosphi2")
        bl = {k: p.get(k) for k in keys}
        bl["nbl"], bl["cosphi"] = p.nbl, p.cosphi
        t0, tl = p.seg_plan()
        n_half = p.n_half
    del B
    assert rep["error_flags"] == 0
    assert rep["s1_counters"][3] == npix * n_half and rep["stage1_terms"] == npix * n_half
    # geometry of the source and its neighbours (bit-identical to the upstream kernel's)
    g = [zeros(9) for _ in range(3)]
    vb.check(vb.lib().vb_pix2lmn_nest(nside, src - 4, 9, g[0].ptr, g[1].ptr, g[2].ptr, None))
    l, m, n = (get(a) for a in g)
    one = dict(B=np.ones(1, np.float32), l=l[4:5], m=m[4:5], n=n[4:5])
    Vo = orc.stage1(one, bl, phase_corrected=1, precision=1)
    emax, erms = rel_err(V, Vo)
    assert emax <= TOL and erms <= TOL, (emax, erms)
    mag = np.hypot(V[0::2], V[1::2])
    seen = mag > 0.5
    assert seen.any() and (~seen).any()                    # both visible and occluded baselines
    assert np.abs(mag[seen] - 1.0).max() < 1e-5 and mag[~seen].max() == 0.0
    sky9 = dict(l=l, m=m, n=n)
    Co, Wo, _ = orc.stage2(sky9, bl, V, t0, tl, mirror=1, blockage=1, occ_mode=2, bl_max=rep["bl_max_m"],
                           lam=kw["lambda_m"], grid_res=kw["grid_res"], precision=1)
    emax, erms = rel_err(Cout[src - 4:src + 5], Co)
    assert emax <= TOL and erms <= TOL, (emax, erms)
