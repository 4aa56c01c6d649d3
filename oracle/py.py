"""ctypes access to the CPU oracle (liboracle.so) and to the upstream
reference harness (oracle/_ref/libref_root.so, libref_vf.so).

Test infrastructure only (see oracle/__init__.py).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_ROOT_SO = HERE / "_ref" / "libref_root.so"
REF_VF_SO = HERE / "_ref" / "libref_vf.so"

vp = C.c_void_p
i64 = C.c_int64
f32 = C.c_float

_or = None
_rr = None
_rv = None


def build_oracle() -> None:
    subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)


def oracle() -> C.CDLL:
    global _or
    if _or is None:
        if not ORACLE_SO.exists():
            build_oracle()
        L = C.CDLL(str(ORACLE_SO))
        sig = {
            "or_num_threads": (C.c_int, []),
            "or_set_threads": (None, [C.c_int]),
            "or_nest_ints": (None, [C.c_int, i64, i64] + [vp] * 7),
            "or_nest_lmn_f64": (None, [C.c_int, i64, i64, vp, vp, vp]),
            "or_occlusion_mask": (None, [i64, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, f32, C.c_int, vp]),
            "or_stage1": (None, [i64, vp, vp, vp, vp, C.c_int, C.c_int] + [vp] * 13 + [f32, C.c_int, C.c_int,
                                                                                      C.c_int, vp, C.c_int,
                                                                                      C.c_int, vp]),
            "or_stage1_subset": (None, [i64, vp, vp, vp, vp, C.c_int] + [vp] * 11 + [f32, C.c_int, C.c_int, vp,
                                                                                    vp]),
            "or_phase_correct_expand": (None, [vp, vp, C.c_int, C.c_int, C.c_int, vp, vp]),
            "or_fa_fb": (None, [vp, vp, vp, C.c_int, vp, vp, vp]),
            "or_grid_params": (None, [f32, f32, f32, f32, C.c_int, vp, vp, vp]),
            "or_keys": (None, [vp, vp, C.c_int, C.c_int, C.c_int, f32, C.c_int, C.c_int, C.c_int, vp]),
            "or_groups": (C.c_int, [vp, C.c_int, vp, vp, vp]),
            "or_stage2": (None, [i64, vp, vp, vp, C.c_int, C.c_int, vp, vp] + [vp] * 13 + [f32, vp, C.c_int,
                                                                                         C.c_int, C.c_int, f32,
                                                                                         f32, C.c_int, C.c_int,
                                                                                         C.c_int, C.c_int, vp,
                                                                                         vp, vp, vp, vp, vp, vp,
                                                                                         vp, vp]),
            "or_stage2_subset": (None, [i64, vp, vp, vp, C.c_int, C.c_int, vp, vp] + [vp] * 11 + [f32, vp, f32,
                                                                                                f32, C.c_int,
                                                                                                C.c_int,
                                                                                                C.c_int, vp,
                                                                                                vp]),
            "or_stage1_subset_simd": (None, [i64, vp, vp, vp, vp, C.c_int] + [vp] * 13 + [f32, C.c_int, vp, vp]),
            "or_stage2_subset_simd": (C.c_int, [i64, vp, vp, vp, C.c_int, C.c_int, vp, vp] + [vp] * 13
                                      + [f32, vp, f32, f32, C.c_int, C.c_int, vp, vp, vp, vp]),
            "or_reference_plan": (None, [f32, vp, vp, vp]),
            "or_window_starts": (None, [f32, C.c_int, C.c_uint64, vp]),
            "or_make_sky": (None, [C.c_int, C.c_uint64, C.c_int, f32, vp]),
            "or_syn_baselines": (None, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_uint64, C.c_int, f32] + [vp] * 11),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _or = L
    return _or


def ref_available() -> bool:
    return REF_ROOT_SO.exists() and REF_VF_SO.exists()


def _sig(L, table):
    for name, (res, args) in table.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


_P = C.c_void_p
_I = C.c_int
_F = C.c_float
_LL = C.c_longlong


def ref_root() -> C.CDLL:
    """Upstream root variant (viss_recon_kernel.cuh, orbit_online.cuh, common.hpp)."""
    global _rr
    if _rr is None:
        L = C.CDLL(str(REF_ROOT_SO))
        _sig(L, {
            "ref_pix2lmn": (_I, [_I, C.c_uint, _I, _P, _P, _P]),
            "ref_invnorm3": (_I, [_P, _P, _P, _P, _I]),
            "ref_orbit": (_I, [_F, _I, C.c_ulonglong, _I, _I] + [_P] * 10),
            "ref_validate_halfsym": (_I, [_P, _P, _P, _I]),
            "ref_viss_halfsym": (_I, [_P, _P, _P, _P, _LL] + [_P] * 11 + [_I, _F, _P]),
            "ref_fa_fb": (None, [_P, _P, _P, _I, _P, _P, _P]),
            "ref_phase_correct_expand": (None, [_P, _P, _I, _P, _P]),
            "ref_locg_full": (_I, [_P, _P, _P, _I, _F, _I, _I]),
            "ref_groups_full": (_I, [_P, _P, _P, _I, _F, _I, _I, _I, _P, _P, _P, _P, _P]),
            "ref_recon_blockage": (_I, [_LL, _P, _P, _P, _P, _P, _P, _P] + [_P] * 8 + [_I, _I, _I, _F, _F, _F, _F,
                                                                                       _I, _P, _P]),
            "ref_recon_keys_avg": (_I, [_LL, _P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _P]),
            "ref_add_normalize": (_I, [_P, _P, _LL]),
            "ref_malloc": (_P, [C.c_size_t]),
            "ref_free": (_I, [_P]),
            "ref_h2d": (_I, [_P, _P, C.c_size_t]),
            "ref_d2h": (_I, [_P, _P, C.c_size_t]),
        })
        _rr = L
    return _rr


def ref_vf() -> C.CDLL:
    """Upstream superset variant (mirror_tile_vissfast)."""
    global _rv
    if _rv is None:
        L = C.CDLL(str(REF_VF_SO))
        _sig(L, {
            "ref_vf_pix2lmn": (_I, [_I, C.c_uint, _I, _P, _P, _P]),
            "ref_vf_nm1": (_I, [_P, _P, _LL]),
            "ref_vf_tile_meta": (_I, [_I, _P, _P, _P, _LL, _P, _P, _P, _P, _P]),
            "ref_vf_classify": (_I, [_P, _P, _P, _F, _I, _P, _P]),
            "ref_vf_viss_tilecone": (_I, [_I, _P, _P, _P, _P, _P, _LL, _P, _P, _P, _P, _P, _I] + [_P] * 11
                                     + [_I, _F, _P]),
            "ref_vf_orbit": (_I, [_F, _I, C.c_ulonglong, _I, _I] + [_P] * 9),
            "ref_vf_locg_half": (_I, [_P, _P, _P, _I, _F, _I, _I]),
            "ref_vf_groups_half": (_I, [_P, _P, _P, _I, _F, _I, _I, _I, _I] + [_P] * 7),
            "ref_vf_recon_rep": (_I, [_LL, _P, _P, _P, _P, _P, _P, _P, _I, _P] + [_P] * 8 + [_F, _F, _F, _P, _P]),
            "ref_vf_recon_half": (_I, [_LL, _P, _P, _P, _P, _P, _P, _P] + [_P] * 8 + [_I, _I, _I, _F, _F, _F, _F,
                                                                                      _I, _P, _P]),
            "ref_vf_recon_keys_avg_half": (_I, [_LL, _P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _P]),
        })
        _rv = L
    return _rv


def ptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


# --- thin numpy wrappers of the oracle -----------------------------------------
def nest_lmn_f64(nside: int, first: int = 0, count: int | None = None):
    """FP64 (l, m, n) of NEST pixels [first, first + count) (default: the whole sky)."""
    n = 12 * nside * nside - first if count is None else count
    l, m, nn = (np.empty(n) for _ in range(3))
    oracle().or_nest_lmn_f64(nside, first, n, ptr(l), ptr(m), ptr(nn))
    return l, m, nn


def nest_ints(nside: int):
    n = 12 * nside * nside
    out = [np.empty(n, dtype=np.int32) for _ in range(7)]
    oracle().or_nest_ints(nside, 0, n, *map(ptr, out))
    return out


def occlusion_mask(l, m, n, x, y, z, invn, cosphi, variant=0, cpe=None):
    npix, nend = l.size, x.size
    out = np.empty(npix * nend, dtype=np.uint8)
    oracle().or_occlusion_mask(npix, ptr(l), ptr(m), ptr(n), nend, ptr(x), ptr(y), ptr(z), ptr(invn), ptr(cpe),
                               float(cosphi), int(variant), ptr(out))
    return out.reshape(nend, npix)


def stage1(sky: dict, bl: dict, *, blockage=1, phase_corrected=1, tile_pix=0, tile_cls=None, precision=1,
           mask_variant=0):
    n_half = bl["u"].size // 2
    V = np.zeros(2 * n_half)
    f = lambda k: ptr(np.ascontiguousarray(bl[k], dtype=np.float32)) if bl.get(k) is not None else None
    keep = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in bl.items() if isinstance(v, np.ndarray)}
    g = lambda k: ptr(keep[k]) if k in keep else None
    oracle().or_stage1(sky["l"].size, ptr(sky["B"]), ptr(sky["l"]), ptr(sky["m"]), ptr(sky["n"]), bl["u"].size,
                       int(bl["nbl"]), g("u"), g("v"), g("w"), g("x1"), g("y1"), g("z1"), g("invn1"), g("x2"),
                       g("y2"), g("z2"), g("invn2"), g("cosphi1"), g("cosphi2"), float(bl["cosphi"]), int(blockage),
                       int(phase_corrected), int(tile_pix), ptr(tile_cls), int(precision), int(mask_variant),
                       ptr(V))
    del f
    return V


def phase_correct_expand(V, w_full, nbl, already=0):
    n_half = V.size // 2
    Vh = np.empty(2 * n_half)
    Vf = np.empty(4 * n_half)
    oracle().or_phase_correct_expand(ptr(V), ptr(w_full), n_half, nbl, already, ptr(Vh), ptr(Vf))
    return Vh, Vf


def fa_fb(u, v, w):
    fa, fb, d = np.zeros(1, np.float32), np.zeros(1, np.float32), np.zeros(1)
    oracle().or_fa_fb(ptr(u), ptr(v), ptr(w), u.size, ptr(fa), ptr(fb), ptr(d))
    return float(fa[0]), float(fb[0]), float(d[0])


def grid_params(fa, fb, bl_max, lam, grid_res=0):
    R, h, du = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.float32)
    oracle().or_grid_params(fa, fb, bl_max, lam, grid_res, ptr(R), ptr(h), ptr(du))
    return int(R[0]), int(h[0]), float(du[0])


def keys(u, v, n, nbl, mirror, inv_du, RES, half, variant=0):
    out = np.empty(n, dtype=np.int32)
    oracle().or_keys(ptr(u), ptr(v), n, nbl, mirror, inv_du, RES, half, variant, ptr(out))
    return out


def groups(k):
    n = k.size
    order, uniq, offs = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n + 1, np.int32)
    nu = oracle().or_groups(ptr(k), n, ptr(order), ptr(uniq), ptr(offs))
    return order, uniq[:nu], offs[:nu + 1]


def stage2(sky: dict, bl: dict, V_half_f32, seg_t0, seg_tlen, *, mirror=1, blockage=1, occ_mode=2, bl_max=100e3,
           lam=30.0, grid_res=0, precision=1, mask_variant=0, key_variant=0, fa=None, fb=None):
    npix = sky["l"].size
    nseg = len(seg_t0)
    keep = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in bl.items() if isinstance(v, np.ndarray)}
    g = lambda k: ptr(keep[k]) if k in keep else None
    t0 = np.ascontiguousarray(seg_t0, dtype=np.int32)
    tl = np.ascontiguousarray(seg_tlen, dtype=np.int32)
    Cc = np.zeros(npix)
    W = np.zeros(npix, dtype=np.uint32)
    sfa, sfb, sdu = (np.zeros(nseg, np.float32) for _ in range(3))
    sR, snu = np.zeros(nseg, np.int32), np.zeros(nseg, np.int32)
    fa_a = None if fa is None else np.ascontiguousarray(fa, dtype=np.float32)
    fb_a = None if fb is None else np.ascontiguousarray(fb, dtype=np.float32)
    Vh = np.ascontiguousarray(V_half_f32, dtype=np.float32)
    oracle().or_stage2(npix, ptr(sky["l"]), ptr(sky["m"]), ptr(sky["n"]), int(bl["nbl"]), nseg, ptr(t0), ptr(tl),
                       g("u"), g("v"), g("w"), g("x1"), g("y1"), g("z1"), g("invn1"), g("x2"), g("y2"), g("z2"),
                       g("invn2"), g("cosphi1"), g("cosphi2"), float(bl["cosphi"]), ptr(Vh), int(mirror),
                       int(blockage), int(occ_mode), float(bl_max), float(lam), int(grid_res), int(precision),
                       int(mask_variant), int(key_variant), ptr(fa_a), ptr(fb_a), ptr(Cc), ptr(W), ptr(sfa),
                       ptr(sfb), ptr(sR), ptr(sdu), ptr(snu))
    return Cc, W, dict(fa=sfa, fb=sfb, RES=sR, du=sdu, nuniq=snu)


def reference_plan(lam):
    a, b, c = (np.zeros(1, np.int32) for _ in range(3))
    oracle().or_reference_plan(lam, ptr(a), ptr(b), ptr(c))
    return int(a[0]), int(b[0]), int(c[0])


def window_starts(lam, day, seed):
    _, pc, _ = reference_plan(lam)
    out = np.zeros(pc, np.int32)
    oracle().or_window_starts(lam, day, seed, ptr(out))
    return out


def make_sky(nside, seed, n_points=20, amp=10.0):
    B = np.empty(12 * nside * nside, np.float32)
    oracle().or_make_sky(nside, seed, n_points, amp, ptr(B))
    return B


def syn_baselines(nsat, T, dt_s=2.0, alt=(400.0, 600.0), spread_km=50.0, R_km=6371.0, seed=42, day=1, lam=30.0):
    nbl = nsat * (nsat - 1) // 2
    n = 2 * nbl * T
    arrs = {k: np.empty(n, np.float32) for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1",
                                                 "invn2")}
    oracle().or_syn_baselines(nsat, T, dt_s, alt[0], alt[1], spread_km, R_km, seed, day, lam,
                              *[ptr(arrs[k]) for k in ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2", "invn1",
                                                       "invn2")])
    arrs["nbl"] = nbl
    return arrs
