"""vb_viss_halfsym_noalloc -- the stage-1 visibility sum for callers that
cannot allocate device memory (hosts whose device memory belongs to another
allocator with a fixed budget, real-time loops that cannot afford the latency
and synchronisation of cudaMalloc) -- against the
workspace entry point vb_viss_halfsym, through the C ABI, on two calls in a
row; the widening of automatic pixel chunks to fit the fixed scratch; its
device error word; and its clear error above the fixed scratch maximum.

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
MAX_BYTES = 64 << 20


def scaled_sky(vb, nside):
    B = vb.synthetic_sky(nside, seed=21)
    return (B.astype(np.float64) * (4 * np.pi / B.size)).astype(np.float32)


def case(vb, nside, tlen, tile=256):
    npix = 12 * nside * nside
    (dl, dm, dn), _ = geometry(nside)
    dB = dev(scaled_sky(vb, nside))
    host, d = reference_baselines(float(np.float32(30.0)), 2, 42, 700, tlen)
    n_full = host["u"].size
    tiles = tile_meta(tile, dl, dm, dn, npix)
    sky = sky_struct(dl, dm, dn, dB, npix, (tile, tiles))
    bl = bl_struct(d, n_full, 28, upstream_cosphi())
    keep = (dl, dm, dn, dB, tiles, d)           # device buffers the structs point into
    return sky, bl, host, d, keep


def noalloc(vb, sky, bl, o, flags=None):
    nh = bl.n_full // 2
    V = zeros(2 * nh, np.float64)
    cnt = zeros(4, np.uint64)
    vb.check(vb.lib().vb_viss_halfsym_noalloc(C.byref(sky), C.byref(bl), C.byref(o), V.ptr, cnt.ptr,
                                              flags.ptr if flags is not None else None, None))
    vb.check(vb.lib().vb_synchronize())
    return get(V, np.float64), get(cnt, np.uint64)


@pytest.mark.parametrize("cull", ["tilecone", "exact", "none"])
def test_noalloc_matches_workspace_entry_point(gpu, vb, cull):
    sky, bl, _, _, keep = case(vb, 32, 24)
    cm = {"tilecone": vb.CULL_TILECONE, "exact": vb.CULL_EXACT, "none": vb.CULL_NONE}[cull]
    V_ref, cnt_ref = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=cm)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=cm, phase_corrected=1, blockage=1)
    for _ in range(2):                      # two calls in a row share the scratch
        V, cnt = noalloc(vb, sky, bl, o)
        emax, erms = rel_err(V, V_ref)
        assert emax <= TOL and erms <= TOL, (emax, erms)
        assert np.array_equal(cnt, cnt_ref)


def test_noalloc_widens_chunks_to_fit(gpu, vb):
    """nside 128 with 57,344 half-baselines: the pixel records fit the fixed
    scratch but the default plan's per-chunk partial sums do not, so the entry
    point widens the pixel chunks.  Staged tiles keep their boundaries, so the
    FP32 tile sums are the same and only the FP64 order across tiles moves:
    V agrees with the workspace entry point to FP64 rounding, and the term
    counters are equal."""
    sky, bl, _, _, keep = case(vb, 128, 2048)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1)
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o))
    assert need > MAX_BYTES, f"default plan needs {need} bytes: the widening path would not run"
    V_ref, cnt_ref = stage1(sky, bl, precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE)
    for _ in range(2):
        V, cnt = noalloc(vb, sky, bl, o)
        emax, erms = rel_err(V, V_ref)
        assert emax <= 1e-10 and erms <= 1e-10, (emax, erms)
        assert np.array_equal(cnt, cnt_ref)


def test_noalloc_keeps_an_explicit_chunk_size(gpu, vb):
    """A chunk size the caller sets is not widened: a plan that does not fit
    with it is rejected."""
    sky, bl, _, _, keep = case(vb, 128, 2048)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1,
                      chunk_pix=256)
    V = zeros(bl.n_full, np.float64)
    rc = vb.lib().vb_viss_halfsym_noalloc(C.byref(sky), C.byref(bl), C.byref(o), V.ptr, None, None, None)
    assert rc == vb._lib.VB_ERR_UNSUPPORTED
    assert b"chunk_pix" in vb.lib().vb_last_error()


def test_noalloc_device_error_word(gpu, vb):
    """The call's device error word comes back through `error_flags`: the
    fp32_fp64phase range bit for a baseline with |u| beyond 2^26 wavelengths,
    the same bit vb_workspace_error_flags reports for the workspace entry
    point, and 0 on the next in-range call (the word in the shared scratch is
    cleared by every call)."""
    sky, bl, host, d, keep = case(vb, 32, 24)
    o = vb.Stage1Opts(precision=vb.PREC_FP32_FP64PH, cull=vb.CULL_TILECONE, phase_corrected=1, blockage=1)
    flags = zeros(1, np.uint32)
    noalloc(vb, sky, bl, o, flags)
    assert int(get(flags, np.uint32)[0]) == 0
    big = host["u"].copy()
    big[5] = np.float32(1.0e8)              # one baseline out of range (finite, no index involved)
    du = dev(big)
    bl.u = du.ptr
    noalloc(vb, sky, bl, o, flags)
    assert int(get(flags, np.uint32)[0]) == 8          # VB_DEVERR_PHASE_RANGE
    need = vb.lib().vb_stage1_workspace_bytes(C.byref(sky), C.byref(bl), C.byref(o))
    ws = zeros(need, np.uint8)
    V = zeros(bl.n_full, np.float64)
    vb.check(vb.lib().vb_viss_halfsym(C.byref(sky), C.byref(bl), C.byref(o), ws.ptr, need, V.ptr, None, None))
    w = C.c_uint(0)
    vb.check(vb.lib().vb_workspace_error_flags(ws.ptr, C.byref(w), None))
    assert w.value == 8
    bl.u = d["u"].ptr
    noalloc(vb, sky, bl, o, flags)
    assert int(get(flags, np.uint32)[0]) == 0


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
    rc = vb.lib().vb_viss_halfsym_noalloc(C.byref(sky), C.byref(bl), C.byref(o), V.ptr, None, None, None)
    assert rc == vb._lib.VB_ERR_UNSUPPORTED
    assert b"maximum" in vb.lib().vb_last_error()
