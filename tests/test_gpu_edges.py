"""Edge cases of the whole pipeline against the FP64 CPU oracle: skies smaller
than one cull tile, one staged pixel block and one stage-2 pixel block;
half-baseline counts that fill no baseline tile; more segments than time
steps; the full (non-mirrored) grid; blockage=0; an all-zero sky.

The upstream code runs the same path at any nside and any orbit length
(main_recon_online.cu:116-134 sizes the day and splits it into segments);
nothing in it special-cases small or ragged sizes, so neither may this build.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err
from test_gpu_pipeline import host_inputs, pipeline_tile_classes

pytestmark = pytest.mark.gpu

TOL = 1e-5

# (nside, nsat, tsteps, segs, mirror, blockage, viss_tile_pix, grid_res)
CASES = {
    "nside1_3sats_5steps": (1, 3, 5, 2, 1, 1, 256, 33),
    "nside2_4sats_7steps_3segs": (2, 4, 7, 3, 1, 1, 256, 33),
    "nside4_full_grid": (4, 5, 9, 2, 0, 1, 64, 65),
    "nside4_blockage0": (4, 5, 9, 2, 1, 0, 64, 65),
    "more_segments_than_steps": (8, 4, 3, 8, 1, 1, 256, 33),
}


def run_case(vb, nside, nsat, tsteps, segs, mirror, blockage, tile, grid_res, B=None):
    cfg = vb.run_config(nside=nside, orbit_model=vb.ORBIT_SYNTHETIC, nsat=nsat, tsteps=tsteps, segs=segs,
                        lambda_m=30.0, occ_R_m=6371e3, cull="tilecone", viss_tile_pix=tile, mirror=mirror,
                        blockage=blockage, grid_res=grid_res, bl_max_m=100e3)
    p = vb.Pipeline(cfg)
    p.set_sky(vb.synthetic_sky(nside, seed=3) if B is None else B)
    p.make_baselines()
    rep = p.run()
    return cfg, p, rep


@pytest.mark.parametrize("case", list(CASES))
def test_small_and_ragged_days_vs_oracle(gpu, vb, orc, case):
    nside, nsat, tsteps, segs, mirror, blockage, tile, grid_res = CASES[case]
    cfg, p, rep = run_case(vb, nside, nsat, tsteps, segs, mirror, blockage, tile, grid_res)
    with p:
        assert rep["error_flags"] == 0
        assert p.npix == 12 * nside * nside
        assert p.n_half == nsat * (nsat - 1) // 2 * tsteps
        Vh, Cd, Wd = p.get("V_half"), p.get("C"), p.get("W")
        sky, bl = host_inputs(p)
        # blockage=0 sums every pixel: no tile classes (the pipeline builds no tile meta)
        cls, tpix = pipeline_tile_classes(vb, p) if blockage else (None, 0)
        Vo = orc.stage1(sky, bl, blockage=blockage, phase_corrected=1, tile_pix=tpix, tile_cls=cls, precision=1)
        emax, erms = rel_err(Vh, Vo)
        assert emax <= TOL and erms <= TOL, (emax, erms)
        t0, tl = p.seg_plan()
        assert len(t0) == min(segs, tsteps) and sum(tl) == tsteps
        Co, Wo, osp = orc.stage2(sky, bl, Vh, t0, tl, mirror=mirror, blockage=blockage, occ_mode=2,
                                 bl_max=cfg.bl_max_m, lam=cfg.lambda_m, grid_res=cfg.grid_res, precision=1)
        assert [s["nuniq"] for s in p.seg_params()] == list(osp["nuniq"])
        if blockage:
            assert np.array_equal(Wd, Wo)
        emax, erms = rel_err(Cd, Co)
        assert emax <= TOL and erms <= TOL, (emax, erms)


def test_zero_sky_gives_exact_zeros(gpu, vb):
    """B = 0 everywhere: every V and every C is exactly zero, while W (the
    visible-group counts) does not depend on the sky."""
    nside = 8
    _, p0, _ = run_case(vb, nside, 4, 16, 2, 1, 1, 256, 33, B=np.zeros(12 * nside * nside, np.float32))
    _, p1, _ = run_case(vb, nside, 4, 16, 2, 1, 1, 256, 33)
    with p0, p1:
        assert not np.any(p0.get("V_half"))
        assert not np.any(p0.get("C"))
        assert np.array_equal(p0.get("W"), p1.get("W"))
        assert np.any(p1.get("C"))
