"""Build recipe of libvissb200 (CUDA, sm_100a) and the drop-in executables.

Every translation unit is compiled with the upstream flags (-O3
--use_fast_math, FMA contraction on) so that the float expressions that decide
occlusion masks, tile classes and uv-cell keys lower to the same instructions
as upstream; precision-critical arithmetic in the hot kernels uses explicit
IEEE intrinsics and FP64 instead of relying on flags.

Usage:  python -m viss_optimize_ws_b200.build [--force]
Outputs (in-tree, git-ignored): viss_optimize_ws_b200/libvissb200.so,
viss_optimize_ws_b200/bin/main_recon_online,
viss_optimize_ws_b200/bin/main_recon_online_mirror_tile_vissfast.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build" / "vissb200"
INCLUDE = ROOT / "include"
LIB = PKG / "libvissb200.so"
BIN = PKG / "bin"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "--use_fast_math", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
           "-I", str(INCLUDE), "-I", str(CSRC)]

LIB_SOURCES = ["vb_geom.cu", "vb_stage1.cu", "vb_stage2.cu", "vb_pipeline.cu", "vb_noalloc.cu"]
EXE_SOURCES = ["main_recon_online.cpp"]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    _run([NVCC, *ARCH, *CUFLAGS, *extra, "-c", str(src), "-o", str(obj)])


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    BIN.mkdir(parents=True, exist_ok=True)
    hdrs = _headers()
    srcs = [CSRC / s for s in LIB_SOURCES if (CSRC / s).exists()]
    objs = []
    jobs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for s in srcs:
            o = BUILD / (s.stem + ".o")
            objs.append(o)
            if force or _stale(o, [s, *hdrs]):
                jobs.append(ex.submit(_compile, s, o, []))
        for j in jobs:
            j.result()
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-fPIC"])
    # drop-in executables (one source, two default sets)
    exe_src = CSRC / "main_recon_online.cpp"
    if exe_src.exists():
        for name, define in (("main_recon_online", "VB_DEFAULTS_ROOT=1"),
                             ("main_recon_online_mirror_tile_vissfast", "VB_DEFAULTS_VISSFAST=1")):
            out = BIN / name
            if force or _stale(out, [exe_src, *objs, *hdrs]):
                _run([NVCC, *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fopenmp", "-I", str(INCLUDE),
                      "-D" + define, str(exe_src), *map(str, objs), "-o", str(out)])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
