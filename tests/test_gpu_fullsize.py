"""Full-size checks at the metric's own workloads, through the FP64 build of
the same pipeline, the CPU FP64 oracle and size-independent properties:
  - the mixed-precision build is within 1e-5 (normwise max and RMS) of the
    FP64 build for V and C, with identical visible-group counts W, at the
    nside-256, nside-512 (precision sweep) and nside-1024 (128 segments,
    occ_mode 2) workloads; the 99th percentile of the per-element error is
    bounded too;
  - the nside-64 plain-method day, whole, against the CPU FP64 oracle;
  - the 64 uneven segments in one batched graph against the same day run
    segment by segment through the kernel-level C ABI, and against FP64;
  - linearity in the sky: V(a B1 + b B2) = a V(B1) + b V(B2), same for C
    (groups and masks do not depend on the sky);
  - a single-pixel sky gives |V_k| = B or 0 (visible or occluded) for every
    baseline, and the term counters add up."""
from __future__ import annotations

import numpy as np
import pytest

import bench
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5


def run(vb, kw, B):
    with vb.Pipeline(vb.run_config(**kw)) as p:
        p.set_sky(B)
        p.make_baselines()
        r = p.run()
        return p.get("V_half"), p.get("C"), p.get("W"), r


P99_TOL = 1e-4   # per-element errors are ill-conditioned where |x| is small: a looser regression bound


@pytest.mark.parametrize("config", [2, 3, 5])
def test_mixed_vs_fp64_at_full_size(gpu, vb, config):
    kw64 = bench.config_kwargs(config, "fp64")
    B = vb.synthetic_sky(kw64["nside"], seed=1)
    V64, C64, W64, r64 = run(vb, kw64, B)
    V, C, W, r = run(vb, bench.config_kwargs(config), B)
    for a, b, what in ((V, V64, "V"), (C, C64, "C")):
        emax, erms = rel_err(a, b)
        assert emax <= TOL and erms <= TOL, f"config {config} {what}: max {emax:.3e} rms {erms:.3e}"
        p99 = bench.err_report(a, b, what == "V")["p99_elem"]
        assert p99 <= P99_TOL, f"config {config} {what}: per-element p99 {p99:.3e}"
    assert np.array_equal(W, W64)
    assert r["s1_counters"] == r64["s1_counters"]
    # stage 2 classifies the groups per pixel block of 256 x (pixels per
    # thread), 4 by default in the mixed build and 2 in FP64: the same totals,
    # and the same split at equal blocks
    assert r["s2_counters"][3] == r64["s2_counters"][3]
    r2 = run(vb, dict(bench.config_kwargs(config), stage2_ppt=2), B)[3]
    assert r2["s2_counters"] == r64["s2_counters"]
    assert r["error_flags"] == 0 and r64["error_flags"] == 0 and r2["error_flags"] == 0
    for cnt in (r["s1_counters"], r["s2_counters"]):
        assert cnt[0] + cnt[1] + cnt[2] == cnt[3]


def test_linearity_in_the_sky_at_full_size(gpu, vb):
    kw = bench.config_kwargs(2)
    B1 = vb.synthetic_sky(256, seed=1)
    B2 = vb.synthetic_sky(256, seed=2)
    a, b = np.float32(0.75), np.float32(-1.5)
    Bc = (a * B1 + b * B2).astype(np.float32)
    V1, C1, W1, _ = run(vb, kw, B1)
    V2, C2, W2, _ = run(vb, kw, B2)
    Vc, Cc, Wc, _ = run(vb, kw, Bc)
    assert np.array_equal(W1, Wc) and np.array_equal(W2, Wc)
    Vl = float(a) * V1.astype(np.float64) + float(b) * V2.astype(np.float64)
    Cl = float(a) * C1.astype(np.float64) + float(b) * C2.astype(np.float64)
    assert rel_err(Vc, Vl)[1] <= TOL and rel_err(Cc, Cl)[1] <= TOL


def test_single_pixel_sky_at_full_size(gpu, vb):
    """One pixel of brightness 1: every V_k is exp(-2 pi i phase) of that
    pixel or 0, so |V_k| is 1 or 0 to FP32 sincos accuracy; over a few pixels
    spread across the sky both cases occur."""
    kw = bench.config_kwargs(2)
    npix = 12 * 256 * 256
    seen_on = seen_off = 0
    with vb.Pipeline(vb.run_config(**kw)) as p:
        p.make_baselines()
        for pix in (123457, 0, 250000, 400000, 600000, npix - 1):
            B = np.zeros(npix, np.float32)
            B[pix] = 1.0
            vb.check(vb.lib().vb_pipeline_set_sky(p.h, B.ctypes.data, 0))   # no pixel-area scaling
            p.run()
            V = p.get("V_half")
            mag = np.hypot(V[0::2].astype(np.float64), V[1::2].astype(np.float64))
            on = mag > 0.5
            assert np.all(np.abs(mag[on] - 1.0) < 1e-5) and np.all(mag[~on] == 0.0), pix
            seen_on += int(on.sum())
            seen_off += int((~on).sum())
    assert seen_on > 0 and seen_off > 0


def test_plain_method_day_vs_cpu_fp64_oracle(gpu, vb, orc):
    """The nside-64 plain-method day (no tile culling, full grid 256, occ_mode 2,
    4 segments), whole, against the CPU FP64 oracle on the pipeline's own
    inputs: mixed within 1e-5, the FP64 build within 1e-7 (float32 output
    rounding), W identical in both."""
    kw = bench.config_kwargs(1)
    B = vb.synthetic_sky(kw["nside"], seed=1)
    with vb.Pipeline(vb.run_config(**kw)) as p:
        p.set_sky(B)
        p.make_baselines()
        r = p.run()
        sky = {k: p.get(k) for k in ("B", "l", "m", "n")}
        bl = {k: p.get(k) for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1", "invn2", "cosphi1",
                                    "cosphi2")}
        bl = {k: v for k, v in bl.items() if v.size}
        bl["nbl"], bl["cosphi"] = p.nbl, p.cosphi
        t0s, tls = p.seg_plan()
        V, C, W = p.get("V_half"), p.get("C"), p.get("W")
        lam = float(p.cfg.lambda_m)
    # the oracle's whole day: its own FP64 V (stored as float32, as the pipeline
    # stores the phase-corrected half set), then its FP64 stage 2
    Vo = orc.stage1(sky, bl, phase_corrected=1, precision=1)
    Co, Wo, _ = orc.stage2(sky, bl, Vo.astype(np.float32), t0s, tls, mirror=0, blockage=1, occ_mode=2,
                           bl_max=r["bl_max_m"], lam=lam, grid_res=kw["grid_res"], precision=1)
    for a, b, what in ((V, Vo, "V"), (C, Co, "C")):
        emax, erms = rel_err(a, b)
        assert emax <= TOL and erms <= TOL, f"{what}: max {emax:.3e} rms {erms:.3e}"
    assert np.array_equal(W, Wo)
    V64, C64, W64, _ = run(vb, bench.config_kwargs(1, "fp64"), B)
    assert rel_err(V64, Vo)[0] <= 2e-7 and rel_err(C64, Co)[0] <= 2e-7
    assert np.array_equal(W64, Wo)


def test_batched_uneven_segments_vs_per_segment_loop(gpu, vb):
    """64 segments of uneven length in one persistent launch per stage (one
    graph) against the same day run segment by segment through
    vb_viss_halfsym / vb_phase_correct_expand / vb_recon_batched: the combined
    images agree to FP32 partial-sum rounding (3e-6); and the batched day is within 1e-5 of the
    FP64 build with W identical."""
    kw = bench.config_kwargs(4)
    B = vb.synthetic_sky(kw["nside"], seed=1)
    with vb.Pipeline(vb.run_config(**kw)) as p:
        p.set_sky(B)
        p.make_baselines()
        r = p.run()
        assert p.nseg == 64 and r["error_flags"] == 0
        t0s, tls = p.seg_plan()
        assert len(set(int(t) for t in tls)) > 1                 # uneven segments
        Cb, Vb, Wb = p.get("C"), p.get("V_half"), p.get("W")
        loop = bench.per_segment_loop(vb, p, {}, 0)
    emax, erms = rel_err(loop["C"], Cb)
    assert emax <= 3e-6 and erms <= 3e-6, (emax, erms)
    V64, C64, W64, _ = run(vb, bench.config_kwargs(4, "fp64"), B)
    for a, b, what in ((Vb, V64, "V"), (Cb, C64, "C")):
        emax, erms = rel_err(a, b)
        assert emax <= TOL and erms <= TOL, f"{what}: max {emax:.3e} rms {erms:.3e}"
    assert np.array_equal(Wb, W64)
