"""vb_viss_halfsym_noalloc -- the stage-1 visibility sum for callers that
cannot allocate device memory (hosts whose device memory belongs to another
allocator with a fixed budget, real-time loops that cannot afford the latency
and synchronisation of cudaMalloc) -- against the
workspace entry point vb_viss_halfsym, through the C ABI, on two calls in a
row; and its clear error above the fixed scratch maximum.

Kept in a file that pytest collects last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from gpu_util import (bl_struct, dev, geometry, get, reference_baselines, sky_struct, stage1, tile_meta,
                      upstream_cosphi, zeros)

pytestmark = pytest.mark.gpu

TOL = 1e-12     # same kernel and plan as the workspace entry point: identical up to this bound


def scaled_sky(vb, nside):
    B = vb.synthetic_sky(nside, seed=21)
    return (B.astype(np.float64) * (4 * np.pi / B.size)).astype(np.float32)


@pytest.mark.parametrize("cull", ["tilecone", "exact", "none"])
def test_noalloc_matches_workspace_entry_point(gpu, vb, cull):
    nside = 32
    npix = 12 * nside * nside
    (dl, dm, dn), _ = geometry(nside)
    dB = dev(scaled_sky(vb, nside))
    host, d = reference_baselines(float(np.float32(30.0)), 2, 42, 700, 24)
    n_full = host["u"].size
    tiles = tile_meta(256, dl, dm, dn, npix)
    sky = sky_struct(dl, dm, dn, dB, npix, (256, tiles))
    bl = bl_struct(d, n_full, 28, upstream_cosphi())
    cm = {"tilecone": vb.CULL_TILECONE, "exact": vb.CULL_EXACT, "none": vb.CULL_NONE}[cull]
    V_ref, cnt_ref = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=cm)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=cm, phase_corrected=1, blockage=1)
    nh = n_full // 2
    for _ in range(2):                      # two calls in a row share the scratch
        V = zeros(2 * nh, np.float64)
        cnt = zeros(4, np.uint64)
        vb.check(vb.lib().vb_viss_halfsym_noalloc(C.byref(sky), C.byref(bl), C.byref(o), V.ptr, cnt.ptr, None))
        vb.check(vb.lib().vb_synchronize())
        emax, erms = rel_err(get(V, np.float64), V_ref)
        assert emax <= TOL and erms <= TOL, (emax, erms)
        assert np.array_equal(get(cnt, np.uint64), cnt_ref)


def test_noalloc_rejects_sizes_beyond_maximum(gpu, vb):
    nside = 512                             # 3.1 M pixels: records alone exceed 64 MiB
    npix = 12 * nside * nside
    (dl, dm, dn), _ = geometry(nside)
    dB = zeros(npix)
    host, d = reference_baselines(float(np.float32(30.0)), 1, 42, 0, 4)
    sky = sky_struct(dl, dm, dn, dB, npix)
    bl = bl_struct(d, host["u"].size, 28, upstream_cosphi())
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_NONE, phase_corrected=1, blockage=1)
    V = zeros(host["u"].size, np.float64)
    rc = vb.lib().vb_viss_halfsym_noalloc(C.byref(sky), C.byref(bl), C.byref(o), V.ptr, None, None)
    assert rc == vb._lib.VB_ERR_UNSUPPORTED
    assert b"maximum" in vb.lib().vb_last_error()
