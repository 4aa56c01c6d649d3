"""The C ABI library loads and exports every entry point include/vissb200.h
declares (no compute calls: runs without a GPU)."""
from __future__ import annotations

import re
import subprocess

from conftest import ROOT


def declared_symbols() -> list[str]:
    text = (ROOT / "include" / "vissb200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(vb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("vb_viss_halfsym", "vb_recon_batched", "vb_pipeline_run", "vb_pix2lmn_nest",
                 "vb_tile_cone_meta", "vb_orbit_make_segment", "vb_fa_fb_host"):
        assert must in names


def test_library_exports_every_declared_symbol(vb):
    lib = vb.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_library_exports_match_nm(vb):
    from viss_optimize_ws_b200._lib import LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (vb_[a-z0-9_]+)", out))
    assert set(declared_symbols()) <= exported


def test_error_strings_without_gpu(vb):
    lib = vb.lib()
    assert lib.vb_error_string(0) == b"ok"
    assert lib.vb_error_string(6).startswith(b"uvw")
    assert lib.vb_version() >= 10000


def test_host_only_entry_points(vb):
    import ctypes as C
    import numpy as np
    lib = vb.lib()
    # long-double plane fit of an exact plane w = 0.25 u - 0.5 v
    rng = np.random.default_rng(1)
    u = rng.uniform(-1000, 1000, 512).astype(np.float32)
    v = rng.uniform(-1000, 1000, 512).astype(np.float32)
    w = (np.float32(0.25) * u - np.float32(0.5) * v).astype(np.float32)
    fa, fb, d = C.c_float(), C.c_float(), C.c_double()
    assert lib.vb_fa_fb_host(u.ctypes.data, v.ctypes.data, w.ctypes.data, u.size, C.byref(fa), C.byref(fb),
                             C.byref(d)) == 0
    assert abs(fa.value - 0.25) < 1e-6 and abs(fb.value + 0.5) < 1e-6
    R, h, du = C.c_int(), C.c_int(), C.c_float()
    assert lib.vb_grid_params(0.0, 0.0, 100e3, 30.0, 0, C.byref(R), C.byref(h), C.byref(du)) == 0
    assert R.value % 2 == 1 and h.value == (R.value - 1) // 2
    assert lib.vb_grid_params(0.0, 0.0, 100e3, 30.0, 512, C.byref(R), C.byref(h), C.byref(du)) == 0
    assert R.value == 513
    # invalid arguments return codes, never exit
    assert lib.vb_grid_params(0.0, 0.0, 100e3, -1.0, 0, C.byref(R), C.byref(h), C.byref(du)) == 1
    B = np.empty(12 * 4 * 4, np.float32)
    assert lib.vb_make_synthetic_sky(4, 3, 2, 10.0, B.ctypes.data) == 0
    assert B.min() >= 0 and B.max() >= 10.0


def test_struct_layouts_match_bindings(vb):
    """Every public struct has the size the ctypes binding assumes (a layout
    slip would pass garbage through the ABI)."""
    import ctypes as C
    from viss_optimize_ws_b200._lib import ABI_STRUCTS
    lib = vb.lib()
    for name, cls in ABI_STRUCTS.items():
        assert lib.vb_abi_sizeof(name.encode()) == C.sizeof(cls), name
    assert lib.vb_abi_sizeof(b"no_such_struct") == 0
    # every typedef'd struct of the header is covered
    text = (ROOT / "include" / "vissb200.h").read_text()
    declared = set(re.findall(r"}\s*(vb_[a-z0-9_]+)\s*;", text))
    assert declared == set(ABI_STRUCTS), declared ^ set(ABI_STRUCTS)


def test_plain_c_caller_compiles_links_and_runs(tmp_path, vb):
    """The header is plain C (a cgo / FFI binding includes it as such): a C99
    program that includes it, links libvissb200 and calls the host-only entry
    points builds with -Wall -Werror and runs without a GPU."""
    from viss_optimize_ws_b200._lib import LIB_PATH
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "vissb200.h"
int main(void) {
  vb_run_config c;
  vb_run_config_defaults(&c);
  if (c.nm1_fast != 1 || c.use_graph != 1) return 2;
  if (vb_abi_sizeof("vb_run_config") != sizeof(vb_run_config)) return 3;
  if (vb_abi_sizeof("vb_stage1_opts") != sizeof(vb_stage1_opts)) return 4;
  if (vb_abi_sizeof("vb_report") != sizeof(vb_report)) return 5;
  int R = 0, half = 0; float du = 0.f;
  if (vb_grid_params(0.f, 0.f, 100e3f, 30.f, 0, &R, &half, &du) != VB_OK) return 6;
  if (vb_run(NULL, NULL, 1, 0, NULL, NULL, NULL) != VB_ERR_INVALID) return 7;
  printf("%d %d %s\n", R, half, vb_error_string(VB_ERR_INVALID));
  return 0;
}
''')
    exe = tmp_path / "caller"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(src),
                        "-o", str(exe), "-L", str(LIB_PATH.parent), "-lvissb200",
                        f"-Wl,-rpath,{LIB_PATH.parent}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.returncode, run.stderr)
    R, half, msg = run.stdout.split(maxsplit=2)
    assert int(R) % 2 == 1 and int(half) == (int(R) - 1) // 2 and msg.strip()
