"""B200-native two-stage direct-sum pipeline (stage 1 visibilities, stage 2
segmented reconstruction) -- Python host glue over the C ABI in
include/vissb200.h.

The compute lives in libvissb200.so (CUDA, sm_100a); this module only moves
numpy arrays in and out and mirrors the upstream run configuration
(main_recon_online.cu flags).  Importing it does not require a GPU; calls
that launch work raise VbError when no device is present.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (CULL_EXACT, CULL_NONE, CULL_TILECONE, ORBIT_REFERENCE, ORBIT_SYNTHETIC, PREC_FP32_DSPH,
                   PREC_FP32_FP64PH, PREC_FP64, PREC_REF32, Baselines, DeviceBuffer, OrbitParams, Report, TuneReport,
                   RunConfig, SegParams, Sky, Stage1Opts, Stage2Opts, VbError, check, download, lib)

__all__ = [
    "lib", "check", "VbError", "DeviceBuffer", "Pipeline", "run_config", "btag_lambda", "synthetic_sky",
    "PREC_REF32", "PREC_FP64", "PREC_FP32_FP64PH", "PREC_FP32_DSPH", "CULL_NONE", "CULL_TILECONE",
    "CULL_EXACT", "ORBIT_REFERENCE", "ORBIT_SYNTHETIC", "Sky", "Baselines", "Stage1Opts", "Stage2Opts",
    "SegParams", "OrbitParams", "RunConfig", "Report",
]

PRECISIONS = {"ref32": PREC_REF32, "fp64": PREC_FP64, "fp32_fp64phase": PREC_FP32_FP64PH,
              "fp32_dsphase": PREC_FP32_DSPH}
CULLS = {"none": CULL_NONE, "tilecone": CULL_TILECONE, "exact": CULL_EXACT}


def btag_lambda(btag: str) -> float:
    """Wavelength (m) of an upstream --btag (main_recon_online.cu:88-89)."""
    f = {"1M": 1e6, "10M": 1e7, "30M": 3e7}[btag]
    return float(np.float32(np.float32(3e8) / np.float32(f)))


def run_config(**kw) -> RunConfig:
    """vb_run_config with library defaults, overridden by keyword arguments."""
    c = RunConfig()
    lib().vb_run_config_defaults(C.byref(c))
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = PRECISIONS[v]
        if k in ("cull", "stage2_cull") and isinstance(v, str):
            v = CULLS[v]
        if not hasattr(c, k):
            raise KeyError(f"unknown run-config field {k!r}")
        setattr(c, k, v)
    return c


def synthetic_sky(nside: int, seed: int = 1, n_points: int = 20, amp: float = 10.0) -> np.ndarray:
    """Seeded sky in NEST order: U[0,1) plus point sources (vb_make_synthetic_sky)."""
    B = np.empty(12 * nside * nside, dtype=np.float32)
    check(lib().vb_make_synthetic_sky(int(nside), int(seed), int(n_points), float(amp), B.ctypes.data))
    return B


class Pipeline:
    """One main_recon_online run context (vb_pipeline)."""

    def __init__(self, cfg: RunConfig | None = None, **kw):
        self.cfg = cfg if cfg is not None else run_config(**kw)
        h = C.c_void_p()
        check(lib().vb_pipeline_create(C.byref(self.cfg), C.byref(h)))
        self.h = h.value
        npix = C.c_int64()
        nseg, nh, nbl, nt = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        cp = C.c_float()
        check(lib().vb_pipeline_info(self.h, C.byref(npix), C.byref(nseg), C.byref(nh), C.byref(nbl),
                                     C.byref(nt), C.byref(cp)))
        self.npix, self.nseg, self.n_half, self.nbl, self.ntile = npix.value, nseg.value, nh.value, nbl.value, nt.value
        self.cosphi = cp.value

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().vb_pipeline_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_sky(self, B: np.ndarray, scale: bool = True) -> None:
        B = np.ascontiguousarray(B, dtype=np.float32)
        if B.size != self.npix:
            raise ValueError(f"sky has {B.size} pixels, expected {self.npix}")
        check(lib().vb_pipeline_set_sky(self.h, B.ctypes.data, int(scale)))

    def make_baselines(self) -> None:
        check(lib().vb_pipeline_make_baselines(self.h))

    def run(self) -> dict:
        r = Report()
        check(lib().vb_pipeline_run(self.h, C.byref(r)))
        return r.as_dict()

    def autotune(self, reps: int = 2) -> dict:
        """vb_pipeline_autotune: fastest kernel shapes for this workload, kept
        in the pipeline's config."""
        t = TuneReport()
        check(lib().vb_pipeline_autotune(self.h, int(reps), C.byref(t)))
        return t.as_dict()

    def run_host(self, B: np.ndarray, scale: bool = True, want_v: bool = False):
        B = np.ascontiguousarray(B, dtype=np.float32)
        Cout = np.empty(self.npix, dtype=np.float32)
        V = np.empty(2 * self.n_half, dtype=np.float32) if want_v else None
        r = Report()
        check(lib().vb_pipeline_run_host(self.h, B.ctypes.data, int(scale), Cout.ctypes.data,
                                         V.ctypes.data if V is not None else None, C.byref(r)))
        return Cout, V, r.as_dict()

    def ptr(self, name: str) -> tuple[int, int]:
        p = C.c_void_p()
        n = C.c_int64()
        check(lib().vb_pipeline_device_ptr(self.h, name.encode(), C.byref(p), C.byref(n)))
        return p.value, n.value

    def get(self, name: str) -> np.ndarray:
        dt = {"C": np.float32, "W": np.uint32, "V_half_d": np.float64, "seg_t0": np.int32,
              "seg_tlen": np.int32}.get(name, np.float32)
        p, n = self.ptr(name)
        if not p or n == 0:
            return np.empty(0, dtype=dt)
        return download(p, dt, n)

    def seg_plan(self) -> tuple[np.ndarray, np.ndarray]:
        t0 = np.empty(self.nseg, dtype=np.int32)
        tl = np.empty(self.nseg, dtype=np.int32)
        check(lib().vb_pipeline_seg_plan(self.h, t0.ctypes.data, tl.ctypes.data))
        return t0, tl

    def seg_params(self) -> list[dict]:
        arr = (SegParams * self.nseg)()
        check(lib().vb_pipeline_seg_params(self.h, arr))
        return [{k: getattr(a, k) for k, _ in SegParams._fields_ if k != "pad"} for a in arr]
