"""Full-size checks at the metric's own workloads (the nside-256 headline
configuration and the nside-512 precision-sweep configuration), through
size-independent properties and the FP64 build of the same pipeline:
  - the mixed-precision build is within 1e-5 (normwise max and RMS) of the
    FP64 build for V and C, with identical visible-group counts W;
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


@pytest.mark.parametrize("config", [2, 3])
def test_mixed_vs_fp64_at_full_size(gpu, vb, config):
    kw64 = bench.config_kwargs(config, "fp64")
    B = vb.synthetic_sky(kw64["nside"], seed=1)
    V64, C64, W64, r64 = run(vb, kw64, B)
    V, C, W, r = run(vb, bench.config_kwargs(config), B)
    for a, b, what in ((V, V64, "V"), (C, C64, "C")):
        emax, erms = rel_err(a, b)
        assert emax <= TOL and erms <= TOL, f"config {config} {what}: max {emax:.3e} rms {erms:.3e}"
    assert np.array_equal(W, W64)
    assert r["s1_counters"] == r64["s1_counters"] and r["s2_counters"] == r64["s2_counters"]
    assert r["error_flags"] == 0 and r64["error_flags"] == 0
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
