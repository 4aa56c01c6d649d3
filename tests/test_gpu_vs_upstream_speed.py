"""Speed against the upstream kernels on the same B200 and the same inputs
(the headline nside-256 workload): the upstream FP32 tile-cone stage-1 kernel
(viss_partial_all_halfsym_tilecone<1024,true>) and the upstream occ_mode=2
representative recon kernel (recon_seg_blockage_half_rep<64>, one launch per
segment, group building not timed), both compiled from the upstream sources
into oracle/_ref, against this build's stage kernels.  Run with -s to see the
times; the test fails if this build is not faster."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

import bench
from gpu_util import dev, vp, zeros

pytestmark = pytest.mark.gpu


def _best(fn, reps=4):
    ts = []
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t)
    return min(ts[1:]) * 1e3


def test_faster_than_upstream_kernels(gpu, vb, ref, record_property):
    kw = bench.workload_kwargs()
    p = vb.Pipeline(vb.run_config(**kw))
    p.set_sky(vb.synthetic_sky(256, seed=1))
    p.make_baselines()
    p.run()
    r = min((p.run() for _ in range(5)), key=lambda x: x["t_s1_kernel_ms"] + x["t_stage2_ms"])
    R = ref.ref_vf()
    P = lambda name: C.c_void_p(p.ptr(name)[0])
    nh, npix = p.n_half, p.npix
    # --- stage 1: upstream tile-cone kernel (its own tile meta at 1024 pixels)
    tile = 1024
    ntile = npix // tile
    meta = [zeros(ntile) for _ in range(5)]
    assert R.ref_vf_tile_meta(tile, P("l"), P("m"), P("n"), C.c_longlong(npix), *[vp(m) for m in meta]) == 0
    Vp = zeros(2 * nh)
    args = [tile, P("B"), P("l"), P("m"), P("n"), P("nm1"), C.c_longlong(npix), *[vp(m) for m in meta], ntile,
            P("u"), P("v"), P("w"), P("x1"), P("y1"), P("z1"), P("invn1"), P("x2"), P("y2"), P("z2"), P("invn2"), nh,
            C.c_float(p.cosphi), vp(Vp)]
    up1 = _best(lambda: R.ref_vf_viss_tilecone(*args))
    # --- stage 2: upstream representative recon, one launch per segment
    sp = p.seg_params()
    t0s, tls = p.seg_plan()
    Vh = P("V_half")
    Cseg, Wseg = zeros(npix), zeros(npix, np.uint32)
    calls, keep = [], []
    for s, (t0, tl) in enumerate(zip(t0s, tls)):
        i0, n = 2 * p.nbl * int(t0), 2 * p.nbl * int(tl)
        nk = n // 2
        Rr, half, du = int(sp[s]["RES"]), int(sp[s]["half"]), float(sp[s]["du"])
        nu = np.zeros(1, np.int32)
        ku, cn, of, ix, rp = (np.zeros(nk + 1, np.int32) for _ in range(5))
        va = np.zeros(2 * nk, np.float32)
        du_, dv_ = C.c_void_p(p.ptr("u")[0] + 4 * i0), C.c_void_p(p.ptr("v")[0] + 4 * i0)
        vh = C.c_void_p(p.ptr("V_half")[0] + 4 * i0)
        assert R.ref_vf_groups_half(du_, dv_, vh, nk, C.c_float(du), Rr, half, 1, 2, nu.ctypes.data, ku.ctypes.data,
                                    cn.ctypes.data, of.ctypes.data, ix.ctypes.data, rp.ctypes.data,
                                    va.ctypes.data) == 0
        k = int(nu[0])
        keys = ku[:k].copy()
        U, V = (keys - 1) // Rr, (keys - 1) % Rr
        ugu = ((U - half).astype(np.float32) * np.float32(du)).astype(np.float32)
        vgu = ((V - half).astype(np.float32) * np.float32(du)).astype(np.float32)
        bufs = (dev(keys), dev(ugu), dev(vgu), dev(rp[:k].copy()))
        keep.append(bufs)
        xs = [C.c_void_p(p.ptr(kk)[0] + 4 * i0) for kk in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2", "invn2")]
        calls.append((C.c_longlong(npix), P("l"), P("m"), P("n"), *[vp(b) for b in bufs], k, vh, *xs,
                      C.c_float(sp[s]["fa"]), C.c_float(sp[s]["fb"]), C.c_float(p.cosphi), vp(Cseg), vp(Wseg)))
    up2 = _best(lambda: [R.ref_vf_recon_rep(*a) for a in calls])
    ours1, ours2 = r["t_s1_kernel_ms"], r["t_stage2_ms"]
    p.close()
    msg = (f"SPEED nside256 10MHz 28672 half-baselines: stage 1 upstream FP32 {up1:.2f} ms, this build "
           f"{ours1:.2f} ms ({up1 / ours1:.2f}x); stage 2 upstream {up2:.2f} ms (recon launches only), "
           f"this build {ours2:.2f} ms incl. grouping ({up2 / ours2:.2f}x)")
    print(msg)
    record_property("speed", msg)
    assert ours1 < up1 and ours2 < up2, msg
