"""Generates the golden fixtures of tests/golden/ by running the UPSTREAM code
itself (oracle/_ref/libref_root.so and libref_vf.so, compiled from the
upstream sources with the upstream flags) on a CUDA GPU.  The fixtures pin
the CPU oracle (tests/test_oracle_golden.py).  Inputs are small seeded cases;
the sky comes from the oracle's seeded generator.

Run on a GPU host:  python tests/golden/make_golden.py --out tests/golden
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import py as orp  # noqa: E402

F32 = np.float32
BL = ("u", "v", "w", "x1", "y1", "z1", "x2", "y2", "z2")


class Dev:
    """Device copy of a host array through the harness helpers."""

    def __init__(self, a=None, nbytes=None, dtype=F32):
        R = orp.ref_root()
        R.ref_malloc.restype = C.c_void_p
        R.ref_malloc.argtypes = [C.c_size_t]
        self.dtype = np.dtype(dtype if a is None else a.dtype)
        self.nbytes = int(a.nbytes if a is not None else nbytes)
        self.ptr = R.ref_malloc(self.nbytes)
        assert self.ptr
        if a is not None:
            a = np.ascontiguousarray(a)
            assert R.ref_h2d(C.c_void_p(self.ptr), a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)) == 0

    def get(self, dtype=None, n=None):
        dt = np.dtype(dtype or self.dtype)
        n = self.nbytes // dt.itemsize if n is None else n
        out = np.empty(n, dt)
        assert orp.ref_root().ref_d2h(out.ctypes.data_as(C.c_void_p), C.c_void_p(self.ptr), C.c_size_t(out.nbytes)) == 0
        return out

    def at(self, byte_off=0):
        return C.c_void_p(self.ptr + byte_off)

    @property
    def p(self):
        return C.c_void_p(self.ptr)


def upstream_cosphi() -> float:
    R, h = F32(1737.1e3), F32(300e3)
    theta = np.arcsin(F32(R / (R + h)), dtype=F32)
    return float(np.cos(F32(np.pi) - theta, dtype=F32))


def orbit(lam, day, seed, t0, tlen):
    n = 56 * tlen
    o = {k: np.zeros(n, F32) for k in BL}
    plan = np.zeros(3, np.int32)
    assert orp.ref_root().ref_orbit(C.c_float(lam), day, C.c_ulonglong(seed), t0, tlen,
                                    *[o[k].ctypes.data_as(C.c_void_p) for k in BL],
                                    plan.ctypes.data_as(C.c_void_p)) == 0
    d = {k: Dev(o[k]) for k in BL}
    for s in ("1", "2"):
        inv = Dev(nbytes=4 * n)
        assert orp.ref_root().ref_invnorm3(d["x" + s].p, d["y" + s].p, d["z" + s].p, inv.p, n) == 0
        d["invn" + s] = inv
        o["invn" + s] = inv.get()
    return o, d, plan


def lmn(nside):
    npix = 12 * nside * nside
    l, m, n = Dev(nbytes=4 * npix), Dev(nbytes=4 * npix), Dev(nbytes=4 * npix)
    assert orp.ref_root().ref_pix2lmn(nside, 0, npix, l.p, m.p, n.p) == 0
    return (l, m, n), (l.get(), m.get(), n.get())


def decode_masks(dl, dm, dn, npix, d, nh, cosphi, tiles=None, tile_pix=256):
    zero = Dev(nbytes=4 * 2 * nh)
    Bblk = Dev((2.0 ** np.arange(16)).astype(F32))
    Vp = Dev(nbytes=8 * nh)
    out = np.zeros((nh, npix), np.uint8)
    nm1 = Dev(nbytes=64)
    for p0 in range(0, npix, 16):
        off = 4 * p0
        if tiles is None:
            rc = orp.ref_root().ref_viss_halfsym(Bblk.p, dl.at(off), dm.at(off), dn.at(off), C.c_longlong(16),
                                                 zero.p, zero.p, zero.p, *[d[k].p for k in ("x1", "y1", "z1", "invn1",
                                                                                            "x2", "y2", "z2", "invn2")],
                                                 nh, C.c_float(cosphi), Vp.p)
        else:
            t = p0 // tile_pix
            rc = orp.ref_vf().ref_vf_viss_tilecone(tile_pix, Bblk.p, dl.at(off), dm.at(off), dn.at(off), nm1.p,
                                                   C.c_longlong(16), *[a.at(4 * t) for a in tiles], 1, zero.p, zero.p,
                                                   zero.p, *[d[k].p for k in ("x1", "y1", "z1", "invn1", "x2", "y2",
                                                                              "z2", "invn2")],
                                                   nh, C.c_float(cosphi), Vp.p)
        assert rc == 0
        vx = Vp.get(F32)[0::2].astype(np.int64)
        for k in range(16):
            out[:, p0 + k] = (vx >> k) & 1
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    cp = upstream_cosphi()

    # --- geometry: l, m, n and tile cones ------------------------------------
    geo = {}
    for nside in (4, 16):
        _, (l, m, n) = lmn(nside)
        geo[f"l{nside}"], geo[f"m{nside}"], geo[f"n{nside}"] = l, m, n
    np.savez_compressed(out / "ref_geometry.npz", **geo)

    # --- orbit: two bands -----------------------------------------------------
    orb = {}
    for tag, (lam, day, seed, t0, tlen) in {"b1M": (300.0, 1, 42, 2000, 16), "b30M": (10.0, 5, 7, 100000, 4)}.items():
        o, _, plan = orbit(float(F32(lam)), day, seed, t0, tlen)
        for k, v in o.items():
            orb[f"{tag}_{k}"] = v
        orb[f"{tag}_plan"] = plan
        orb[f"{tag}_args"] = np.array([lam, day, seed, t0, tlen], np.float64)
    np.savez_compressed(out / "ref_orbit.npz", **orb)

    # --- stage 1: nside 16, 1M band, 16 steps ---------------------------------
    nside, lam = 16, float(F32(300.0))
    npix = 12 * nside * nside
    (dl, dm, dn), (l, m, n) = lmn(nside)
    B = orp.make_sky(nside, 3)
    B = (B.astype(np.float64) * (4 * np.pi / npix)).astype(F32)
    dB = Dev(B)
    o, d, _ = orbit(lam, 1, 42, 2000, 16)
    nh = o["u"].size // 2
    Vp = Dev(nbytes=8 * nh)
    assert orp.ref_root().ref_viss_halfsym(dB.p, dl.p, dm.p, dn.p, C.c_longlong(npix), d["u"].p, d["v"].p, d["w"].p,
                                           *[d[k].p for k in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2", "invn2")],
                                           nh, C.c_float(cp), Vp.p) == 0
    V_plain = Vp.get(F32)
    tiles = [Dev(nbytes=4 * (npix // 256)) for _ in range(5)]
    assert orp.ref_vf().ref_vf_tile_meta(256, dl.p, dm.p, dn.p, C.c_longlong(npix), *[t.p for t in tiles]) == 0
    nm1 = Dev(nbytes=4 * npix)
    assert orp.ref_vf().ref_vf_nm1(dn.p, nm1.p, C.c_longlong(npix)) == 0
    assert orp.ref_vf().ref_vf_viss_tilecone(256, dB.p, dl.p, dm.p, dn.p, nm1.p, C.c_longlong(npix),
                                             *[t.p for t in tiles], npix // 256, d["u"].p, d["v"].p, d["w"].p,
                                             *[d[k].p for k in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2",
                                                                "invn2")], nh, C.c_float(cp), Vp.p) == 0
    V_tile = Vp.get(F32)
    m_plain = decode_masks(dl, dm, dn, npix, d, nh, cp)
    m_tile = decode_masks(dl, dm, dn, npix, d, nh, cp, tiles=tiles)
    s1 = dict(B=B, l=l, m=m, n=n, cosphi=np.array([cp], F32), V_plain=V_plain, V_tile=V_tile,
              mask_plain=np.packbits(m_plain, axis=1), mask_tile=np.packbits(m_tile, axis=1),
              tile=np.stack([t.get() for t in tiles]), **{k: o[k] for k in o})
    np.savez_compressed(out / "ref_stage1.npz", **s1)

    # --- stage 2: 4 segments of 16 steps, mirror rep path and full grid ------------
    o, d, _ = orbit(lam, 1, 42, 100, 64)
    nh = o["u"].size // 2
    Vp = Dev(nbytes=8 * nh)
    assert orp.ref_root().ref_viss_halfsym(dB.p, dl.p, dm.p, dn.p, C.c_longlong(npix), d["u"].p, d["v"].p, d["w"].p,
                                           *[d[k].p for k in ("x1", "y1", "z1", "invn1", "x2", "y2", "z2", "invn2")],
                                           nh, C.c_float(cp), Vp.p) == 0
    Vraw = Vp.get(F32)
    Vh, Vf = np.zeros(2 * nh, F32), np.zeros(4 * nh, F32)
    orp.ref_root().ref_phase_correct_expand(Vraw.ctypes.data_as(C.c_void_p), o["w"].ctypes.data_as(C.c_void_p), nh,
                                            Vh.ctypes.data_as(C.c_void_p), Vf.ctypes.data_as(C.c_void_p))
    dVh, dVf = Dev(Vh), Dev(Vf)
    bl_max = 100e3
    s2 = dict(Vraw=Vraw, V_half=Vh, V_full=Vf, **{k: o[k] for k in o})
    Cacc = {k: np.zeros(npix, np.float64) for k in ("rep", "full2", "full0")}
    Wacc = {k: np.zeros(npix, np.int64) for k in ("rep", "full2", "full0")}
    Cseg, Wseg = Dev(nbytes=4 * npix), Dev(nbytes=4 * npix)
    for s in range(4):
        t0, tl = 16 * s, 16
        i0, nfull = 56 * t0, 56 * tl
        nk = nfull // 2
        fa, fb, den = np.zeros(1, F32), np.zeros(1, F32), np.zeros(1)
        orp.ref_root().ref_fa_fb(o["u"][i0:].ctypes.data_as(C.c_void_p), o["v"][i0:].ctypes.data_as(C.c_void_p),
                                 o["w"][i0:].ctypes.data_as(C.c_void_p), nfull, fa.ctypes.data_as(C.c_void_p),
                                 fb.ctypes.data_as(C.c_void_p), den.ctypes.data_as(C.c_void_p))
        R, half, du = orp.grid_params(float(fa[0]), float(fb[0]), bl_max, lam)
        inv = float(F32(1.0) / F32(du))
        s2[f"s{s}_fa"], s2[f"s{s}_fb"], s2[f"s{s}_denom"] = fa, fb, den
        s2[f"s{s}_grid"] = np.array([R, half], np.int32)
        s2[f"s{s}_du"] = np.array([du], F32)
        # keys (half and full)
        kh, kf = Dev(nbytes=4 * nk), Dev(nbytes=4 * nfull)
        assert orp.ref_vf().ref_vf_locg_half(d["u"].at(4 * i0), d["v"].at(4 * i0), kh.p, nk, C.c_float(inv), R,
                                             half) == 0
        assert orp.ref_root().ref_locg_full(d["u"].at(4 * i0), d["v"].at(4 * i0), kf.p, nfull, C.c_float(inv), R,
                                            half) == 0
        s2[f"s{s}_keys_half"], s2[f"s{s}_keys_full"] = kh.get(np.int32), kf.get(np.int32)
        # half groups with representatives (occ_mode 2) and members (occ_mode 0)
        nu = np.zeros(1, np.int32)
        ku, cn, of, ix, rp = (np.zeros(nk + 1, np.int32) for _ in range(5))
        va = np.zeros(2 * nk, F32)
        ptrs = lambda: [x.ctypes.data_as(C.c_void_p) for x in (nu, ku, cn, of, ix, rp, va)]
        assert orp.ref_vf().ref_vf_groups_half(d["u"].at(4 * i0), d["v"].at(4 * i0), dVh.at(4 * i0), nk,
                                               C.c_float(du), R, half, 1, 2, *ptrs()) == 0
        k = int(nu[0])
        s2[f"s{s}_half_uniq"], s2[f"s{s}_half_counts"], s2[f"s{s}_half_rep"] = ku[:k].copy(), cn[:k].copy(), rp[:k].copy()
        assert orp.ref_vf().ref_vf_groups_half(d["u"].at(4 * i0), d["v"].at(4 * i0), dVh.at(4 * i0), nk,
                                               C.c_float(du), R, half, 1, 0, *ptrs()) == 0
        s2[f"s{s}_half_offsets"], s2[f"s{s}_half_order"] = of[:k + 1].copy(), ix[:nk].copy()
        # mirror representative recon of the segment
        keys = s2[f"s{s}_half_uniq"]
        U, V = (keys - 1) // R, (keys - 1) % R
        ugu = ((U - half).astype(F32) * F32(du)).astype(F32)
        vgu = ((V - half).astype(F32) * F32(du)).astype(F32)
        assert orp.ref_vf().ref_vf_recon_rep(C.c_longlong(npix), dl.p, dm.p, dn.p, Dev(keys).p, Dev(ugu).p,
                                             Dev(vgu).p, Dev(s2[f"s{s}_half_rep"]).p, k, dVh.at(4 * i0),
                                             *[d[kk].at(4 * i0) for kk in ("x1", "y1", "z1", "invn1", "x2", "y2",
                                                                           "z2", "invn2")],
                                             C.c_float(fa[0]), C.c_float(fb[0]), C.c_float(cp), Cseg.p, Wseg.p) == 0
        Cacc["rep"] += Cseg.get(F32)
        Wacc["rep"] += Wseg.get(np.uint32)
        # full grid groups + recon_seg_blockage (occ_mode 2 and 0)
        nuf = np.zeros(1, np.int32)
        kuf, off, ixf = np.zeros(nfull + 1, np.int32), np.zeros(nfull + 1, np.int32), np.zeros(nfull, np.int32)
        vaf = np.zeros(2 * nfull, F32)
        assert orp.ref_root().ref_groups_full(d["u"].at(4 * i0), d["v"].at(4 * i0), dVf.at(8 * i0), nfull,
                                              C.c_float(du), R, half, 1, nuf.ctypes.data_as(C.c_void_p),
                                              kuf.ctypes.data_as(C.c_void_p), off.ctypes.data_as(C.c_void_p),
                                              ixf.ctypes.data_as(C.c_void_p), vaf.ctypes.data_as(C.c_void_p)) == 0
        kf_ = int(nuf[0])
        s2[f"s{s}_full_uniq"], s2[f"s{s}_full_offsets"], s2[f"s{s}_full_order"] = kuf[:kf_].copy(), off[:kf_ + 1].copy(), ixf.copy()
        for occ, tag in ((2, "full2"), (0, "full0")):
            assert orp.ref_root().ref_recon_blockage(C.c_longlong(npix), dl.p, dm.p, dn.p, Dev(kuf[:kf_]).p,
                                                     Dev(off[:kf_ + 1]).p, Dev(ixf).p, dVf.at(8 * i0),
                                                     *[d[kk].at(4 * i0) for kk in ("x1", "y1", "z1", "invn1", "x2",
                                                                                   "y2", "z2", "invn2")],
                                                     kf_, R, half, C.c_float(du), C.c_float(fa[0]), C.c_float(fb[0]),
                                                     C.c_float(cp), occ, Cseg.p, Wseg.p) == 0
            Cacc[tag] += Cseg.get(F32)
            Wacc[tag] += Wseg.get(np.uint32)
    for k in Cacc:
        s2[f"C_{k}"] = np.where(Wacc[k] > 0, Cacc[k] / np.maximum(Wacc[k], 1), 0.0)
        s2[f"W_{k}"] = Wacc[k]
    s2["meta"] = np.array([nside, lam, bl_max, cp], np.float64)
    np.savez_compressed(out / "ref_stage2.npz", **s2)
    for f in sorted(out.glob("ref_*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
