"""ctypes binding of libvissb200 (include/vissb200.h).

The shared library is built in-tree by viss_optimize_ws_b200.build; loading
fails loudly when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libvissb200.so"

VB_OK = 0
VB_ERR_INVALID, VB_ERR_CUDA, VB_ERR_TIMEOUT, VB_ERR_NOMEM = 1, 2, 3, 4
VB_ERR_UNSUPPORTED, VB_ERR_HALFSYM, VB_ERR_IO = 5, 6, 7
PREC_REF32, PREC_FP64, PREC_FP32_FP64PH, PREC_FP32_DSPH = 0, 1, 2, 3
CULL_NONE, CULL_TILECONE, CULL_EXACT = 0, 1, 2
ORBIT_REFERENCE, ORBIT_SYNTHETIC = 0, 1
H2D, D2H, D2D = 0, 1, 2

vp = C.c_void_p
fp = C.POINTER(C.c_float)


class VbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Sky(C.Structure):
    _fields_ = [("npix", C.c_int64), ("B", vp), ("l", vp), ("m", vp), ("n", vp), ("tile_pix", C.c_int),
                ("cx", vp), ("cy", vp), ("cz", vp), ("cosA", vp), ("sinA", vp)]


class Baselines(C.Structure):
    _fields_ = [("n_full", C.c_int), ("nbl", C.c_int), ("u", vp), ("v", vp), ("w", vp),
                ("x1", vp), ("y1", vp), ("z1", vp), ("invn1", vp), ("x2", vp), ("y2", vp), ("z2", vp),
                ("invn2", vp), ("cosphi1", vp), ("cosphi2", vp), ("cosphi", C.c_float)]


class Stage1Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("cull", C.c_int), ("phase_corrected", C.c_int), ("blockage", C.c_int),
                ("bpt", C.c_int), ("stage_pix", C.c_int), ("chunk_pix", C.c_int), ("exact_tile_pix", C.c_int),
                ("ctas_per_sm", C.c_int), ("items_per_cta", C.c_int), ("refine_pix", C.c_int),
                ("mask_visible_tiles", C.c_int)]


class Stage2Opts(C.Structure):
    _fields_ = [("mirror", C.c_int), ("blockage", C.c_int), ("occ_mode", C.c_int), ("precision", C.c_int),
                ("cull", C.c_int), ("grid_res", C.c_int), ("bl_max", C.c_float), ("lambda_", C.c_float),
                ("ppt", C.c_int), ("items_per_cta", C.c_int)]


class SegParams(C.Structure):
    _fields_ = [("fa", C.c_float), ("fb", C.c_float), ("du", C.c_float), ("inv_du", C.c_float),
                ("RES", C.c_int), ("half", C.c_int), ("nuniq", C.c_int), ("group_start", C.c_int),
                ("denom", C.c_double), ("n_keyed", C.c_int), ("pad", C.c_int)]


class OrbitParams(C.Structure):
    _fields_ = [("model", C.c_int), ("lambda_m", C.c_float), ("day", C.c_int), ("seed", C.c_uint64),
                ("nsat", C.c_int), ("tsteps", C.c_int), ("dt_s", C.c_double), ("alt_min_km", C.c_double),
                ("alt_max_km", C.c_double), ("spread_km", C.c_double), ("occ_R_m", C.c_double)]


class RunConfig(C.Structure):
    _fields_ = [("nside", C.c_int), ("day", C.c_int), ("segs", C.c_int), ("blockage", C.c_int),
                ("occ_mode", C.c_int), ("orbit_seed", C.c_uint64), ("lambda_m", C.c_float),
                ("viss_tile_pix", C.c_int), ("mirror", C.c_int), ("cull", C.c_int), ("precision", C.c_int),
                ("orbit_model", C.c_int), ("nsat", C.c_int), ("tsteps", C.c_int), ("dt_s", C.c_double),
                ("alt_min_km", C.c_double), ("alt_max_km", C.c_double), ("spread_km", C.c_double),
                ("occ_R_m", C.c_double), ("bl_max_m", C.c_float), ("grid_res", C.c_int), ("seg_plan", C.c_int),
                ("seg_min_half", C.c_int), ("seg_max_half", C.c_int), ("seg_seed", C.c_uint64),
                ("stage2_cull", C.c_int), ("stage2_ppt", C.c_int), ("stage2_items_per_cta", C.c_int),
                ("stage1_bpt", C.c_int), ("stage1_stage_pix", C.c_int), ("stage1_ctas_per_sm", C.c_int),
                ("stage1_items_per_cta", C.c_int), ("stage1_refine_pix", C.c_int), ("slab_pix", C.c_int64), ("use_graph", C.c_int), ("device", C.c_int),
                ("nm1_fast", C.c_int)]


class Report(C.Structure):
    _fields_ = [("npix_hi", C.c_int), ("npix_lo", C.c_int), ("nseg", C.c_int), ("n_half_total", C.c_int),
                ("stage1_terms", C.c_longlong), ("stage2_terms", C.c_longlong), ("groups_total", C.c_longlong),
                ("t_stage1_ms", C.c_double), ("t_stage2_ms", C.c_double), ("t_orbit_ms", C.c_double),
                ("s1_counters", C.c_ulonglong * 4), ("s2_counters", C.c_ulonglong * 4),
                ("w_scalar_total", C.c_double), ("t_s1_kernel_ms", C.c_double), ("t_s2_kernel_ms", C.c_double),
                ("t_e2e_ms", C.c_double), ("error_flags", C.c_int), ("graph_kernels", C.c_int),
                ("bl_max_m", C.c_double)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("s1_counters", "s2_counters")}
        d["npix"] = (self.npix_hi << 31) | self.npix_lo
        d["s1_counters"] = list(self.s1_counters)
        d["s2_counters"] = list(self.s2_counters)
        return d


class TuneReport(C.Structure):
    _fields_ = [("stage1_bpt", C.c_int), ("stage1_stage_pix", C.c_int), ("stage1_ctas_per_sm", C.c_int),
                ("stage1_items_per_cta", C.c_int), ("stage2_ppt", C.c_int), ("stage2_items_per_cta", C.c_int),
                ("stage1_ms", C.c_double), ("stage2_ms", C.c_double), ("stage1_default_ms", C.c_double),
                ("stage2_default_ms", C.c_double), ("candidates", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


# ctypes mirror of each public struct, checked against vb_abi_sizeof
ABI_STRUCTS = {"vb_sky": Sky, "vb_baselines": Baselines, "vb_stage1_opts": Stage1Opts, "vb_stage2_opts": Stage2Opts,
               "vb_seg_params": SegParams, "vb_orbit_params": OrbitParams, "vb_run_config": RunConfig,
               "vb_report": Report, "vb_tune_report": TuneReport}


_SIGS = {
    "vb_version": (C.c_int, []),
    "vb_error_string": (C.c_char_p, [C.c_int]),
    "vb_last_error": (C.c_char_p, []),
    "vb_device_info": (C.c_int, [C.POINTER(C.c_int)] * 3),
    "vb_pix2lmn_nest": (C.c_int, [C.c_int, C.c_uint32, C.c_int64, vp, vp, vp, vp]),
    "vb_build_nm1": (C.c_int, [vp, vp, C.c_int64, vp]),
    "vb_tile_cone_meta": (C.c_int, [C.c_int, vp, vp, vp, C.c_int64, vp, vp, vp, vp, vp, vp]),
    "vb_classify_tile_cone": (C.c_int, [vp, vp, vp, C.c_float, C.c_int, vp, vp, vp]),
    "vb_invnorm3": (C.c_int, [vp, vp, vp, vp, C.c_int, vp]),
    "vb_occlusion_mask": (C.c_int, [vp, vp, vp, C.c_int64, vp, vp, vp, vp, vp, C.c_float, C.c_int, vp, vp]),
    "vb_orbit_create": (C.c_int, [C.POINTER(OrbitParams), C.POINTER(vp)]),
    "vb_orbit_info": (C.c_int, [vp] + [C.POINTER(C.c_int)] * 5),
    "vb_orbit_make_segment": (C.c_int, [vp, C.c_int, C.c_int] + [vp] * 11 + [vp]),
    "vb_orbit_destroy": (C.c_int, [vp]),
    "vb_validate_uvw_halfsym": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.POINTER(C.c_int), vp]),
    "vb_stage1_workspace_bytes": (C.c_size_t, [C.POINTER(Sky), C.POINTER(Baselines), C.POINTER(Stage1Opts)]),
    "vb_viss_halfsym": (C.c_int, [C.POINTER(Sky), C.POINTER(Baselines), C.POINTER(Stage1Opts), vp, C.c_size_t,
                                  vp, vp, vp]),
    "vb_viss_halfsym_noalloc": (C.c_int, [C.POINTER(Sky), C.POINTER(Baselines), C.POINTER(Stage1Opts), vp, vp,
                                          vp, vp]),
    "vb_stage1_tile_classes": (C.c_int, [C.POINTER(Sky), C.POINTER(Baselines), C.POINTER(Stage1Opts), vp,
                                         C.c_size_t, vp, C.POINTER(C.c_int), vp]),
    "vb_phase_correct_expand": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
    "vb_fa_fb_host": (C.c_int, [vp, vp, vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                C.POINTER(C.c_double)]),
    "vb_grid_params": (C.c_int, [C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "vb_build_keys": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, vp, vp]),
    "vb_stage2_workspace_bytes": (C.c_size_t, [C.c_int, C.c_int, C.c_int64, C.POINTER(Stage2Opts)]),
    "vb_recon_batched": (C.c_int, [C.POINTER(Sky), C.POINTER(Baselines), vp, C.c_int, vp, vp,
                                   C.POINTER(Stage2Opts), vp, C.c_size_t, vp, vp, vp, vp, vp]),
    "vb_stage1": (C.c_int, [C.POINTER(Sky), C.POINTER(Baselines), C.POINTER(Stage1Opts), vp, C.c_size_t, vp,
                            vp]),
    "vb_stage2": (C.c_int, [C.POINTER(Sky), C.POINTER(Baselines), vp, C.c_int, vp, vp, C.POINTER(Stage2Opts),
                            vp, C.c_size_t, vp, vp, vp]),
    "vb_run": (C.c_int, [C.POINTER(RunConfig), vp, C.c_int, C.c_int64, vp, vp, C.POINTER(Report)]),
    "vb_workspace_error_flags": (C.c_int, [vp, C.POINTER(C.c_uint), vp]),
    "vb_run_config_defaults": (None, [C.POINTER(RunConfig)]),
    "vb_pipeline_create": (C.c_int, [C.POINTER(RunConfig), C.POINTER(vp)]),
    "vb_pipeline_set_sky": (C.c_int, [vp, vp, C.c_int]),
    "vb_pipeline_make_baselines": (C.c_int, [vp]),
    "vb_pipeline_run": (C.c_int, [vp, C.POINTER(Report)]),
    "vb_pipeline_run_host": (C.c_int, [vp, vp, C.c_int, vp, vp, C.POINTER(Report)]),
    "vb_pipeline_device_ptr": (C.c_int, [vp, C.c_char_p, C.POINTER(vp), C.POINTER(C.c_int64)]),
    "vb_pipeline_info": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "vb_pipeline_seg_plan": (C.c_int, [vp, vp, vp]),
    "vb_pipeline_seg_params": (C.c_int, [vp, vp]),
    "vb_pipeline_destroy": (C.c_int, [vp]),
    "vb_pipeline_autotune": (C.c_int, [vp, C.c_int, C.POINTER(TuneReport)]),
    "vb_pipeline_set_day": (C.c_int, [vp, C.c_int]),
    "vb_accumulate": (C.c_int, [vp, C.c_int64, vp, vp]),
    "vb_abi_sizeof": (C.c_size_t, [C.c_char_p]),
    "vb_measure_peaks": (C.c_int, [C.POINTER(C.c_double)] * 4),
    "vb_flush_l2": (C.c_int, [vp, C.c_size_t, vp]),
    "vb_set_device": (C.c_int, [C.c_int]),
    "vb_host_alloc": (C.c_int, [C.POINTER(vp), C.c_size_t]),
    "vb_host_free": (C.c_int, [vp]),
    "vb_malloc": (C.c_int, [C.POINTER(vp), C.c_size_t]),
    "vb_free": (C.c_int, [vp]),
    "vb_memcpy": (C.c_int, [vp, vp, C.c_size_t, C.c_int]),
    "vb_memset": (C.c_int, [vp, C.c_int, C.c_size_t]),
    "vb_synchronize": (C.c_int, []),
    "vb_make_synthetic_sky": (C.c_int, [C.c_int, C.c_uint64, C.c_int, C.c_float, vp]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libvissb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m viss_optimize_ws_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != VB_OK:
        msg = lib().vb_last_error().decode(errors="replace")
        raise VbError(rc, msg)


# --- device buffers ------------------------------------------------------------
class DeviceBuffer:
    """Owned device allocation with numpy upload / download."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        p = vp()
        check(lib().vb_malloc(C.byref(p), max(1, self.nbytes)))
        self.ptr = p.value

    @classmethod
    def from_array(cls, a: np.ndarray) -> "DeviceBuffer":
        a = np.ascontiguousarray(a)
        b = cls(a.nbytes)
        if a.nbytes:
            check(lib().vb_memcpy(b.ptr, a.ctypes.data, a.nbytes, H2D))
        return b

    def to_array(self, dtype, count: int | None = None) -> np.ndarray:
        dt = np.dtype(dtype)
        n = self.nbytes // dt.itemsize if count is None else int(count)
        out = np.empty(n, dtype=dt)
        if n:
            check(lib().vb_memcpy(out.ctypes.data, self.ptr, n * dt.itemsize, D2H))
        return out

    def zero(self) -> None:
        check(lib().vb_memset(self.ptr, 0, self.nbytes))

    def free(self) -> None:
        if self.ptr:
            lib().vb_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def download(ptr: int, dtype, count: int) -> np.ndarray:
    out = np.empty(int(count), dtype=np.dtype(dtype))
    if count:
        check(lib().vb_memcpy(out.ctypes.data, ptr, out.nbytes, D2H))
    return out
