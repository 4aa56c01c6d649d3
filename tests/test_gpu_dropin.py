"""The drop-in executables against the upstream executables (built from the
upstream sources into oracle/_ref) with the flag set of the upstream
parameter script (main_recon_online.sh), reduced to a small sky:
identical uvw / xyza / xyzb files, identical per-segment plane fits, grid
sizes and group counts, and V / C that agree to the upstream FP32 level."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu

BIN = ROOT / "viss_optimize_ws_b200" / "bin"
UP = ROOT / "oracle" / "_ref"


def run(exe: Path, args: list[str], cwd: Path) -> subprocess.CompletedProcess:
    r = subprocess.run([str(exe), *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    return r


def seg_lines(out: str) -> list[tuple]:
    rows = []
    for line in out.splitlines():
        if not (line.startswith("[seg ") or line.startswith("[day ")) or "segN=" not in line:
            continue
        d = dict(re.findall(r"(\w+)=([^\s\]\[]+)", line))
        nu = d.get("nuniq", d.get("nuniq_halfgrid"))
        rows.append((int(d["t0"]), int(d["segN"]), d["fa"], d["fb"], int(nu), int(d["RES"])))
    return rows


@pytest.mark.parametrize("variant", ["root", "vissfast"])
def test_dropin_matches_upstream_executable(gpu, vb, tmp_path, variant):
    sky = tmp_path / "sky"
    exe = BIN / ("main_recon_online" if variant == "root" else "main_recon_online_mirror_tile_vissfast")
    up = UP / exe.name
    assert exe.exists() and up.exists()
    common = ["--btag=1M", "--nside=32", "--segs=4", "--blockage=1", "--occ_mode=2", f"--sky_dir={sky}",
              "--gpus=0", "--gen_gpu_index=0", "--B_mode=bin", "--orbit_seed=42", "--write_viss=1",
              "--write_baseline_txt=1"]
    if variant == "root":
        common.append("--day=1")
    else:
        common += ["--day_start=1", "--day_count=1", "--C_mode=txt"]
    mine, theirs = tmp_path / "mine", tmp_path / "up"
    r1 = run(exe, common + [f"--out_dir={mine}/", "--sky_gen=5"], tmp_path)
    assert r1.returncode == 0, r1.stderr
    # upstream's vissfast build reads B_10M.bin / B.bin whatever the btag
    data = (sky / "B_1M.bin").read_bytes()
    (sky / "B_10M.bin").write_bytes(data)
    (sky / "B.bin").write_bytes(data)
    r2 = run(up, common + [f"--out_dir={theirs}/"], tmp_path)
    assert r2.returncode == 0, r2.stderr
    # identical generated baselines (text formatting of identical floats)
    for f in ("uvw1day1M.txt", "xyza1day1M.txt", "xyzb1day1M.txt"):
        if variant == "vissfast" and not (theirs / f).exists():
            continue
        assert (mine / f).read_bytes() == (theirs / f).read_bytes(), f
    # identical per-segment plan numbers
    a, b = seg_lines(r1.stdout), seg_lines(r2.stdout)
    assert len(a) == len(b) == 4
    assert a == b
    # V and C to the upstream FP32 level
    Vm = np.loadtxt(mine / "Viss1day1M.txt")
    Vu = np.loadtxt(theirs / "Viss1day1M.txt")
    assert Vm.shape == Vu.shape
    ev = rel_err(Vu, Vm)
    assert ev[0] < 1e-3 and ev[1] < 1e-3, ev
    Cm = np.loadtxt(mine / "C1day1M.txt")
    Cu = np.loadtxt(theirs / "C1day1M.txt")
    ec = rel_err(Cu, Cm)
    assert ec[0] < 5e-3 and ec[1] < 5e-3, ec


def test_dropin_error_paths(tmp_path):
    exe = BIN / "main_recon_online"
    r = run(exe, ["--btag=7M"], tmp_path)
    assert r.returncode == 1 and "ERROR --btag" in r.stderr
    r = run(exe, ["--btag=1M", "--nside=8", f"--sky_dir={tmp_path}/none", f"--out_dir={tmp_path}/o/"], tmp_path)
    assert r.returncode == 1 and "ERROR" in r.stderr
    # short sky file -> error exit 1 (upstream: load_single_bin_exact size check)
    (tmp_path / "s").mkdir()
    np.zeros(100, np.float32).tofile(tmp_path / "s" / "B_1M.bin")
    r = run(exe, ["--btag=1M", "--nside=8", f"--sky_dir={tmp_path}/s", "--B_mode=bin", f"--out_dir={tmp_path}/o/"],
            tmp_path)
    assert r.returncode == 1 and "ERROR reading B" in r.stderr


def test_parameter_scripts_and_autotune(gpu, vb, tmp_path):
    """The shipped parameter scripts run the drop-in binaries with the
    upstream flag set (values from the environment); --autotune=1 picks kernel
    shapes on the first day and gives the untuned C to summation rounding."""
    import os
    run_dir = ROOT / "viss_optimize_ws_b200" / "run"
    env = dict(os.environ, BTAG="1M", NSIDE="32", SEGS="4", SKY_DIR=str(tmp_path / "sky"), GPUS="0")
    outs = {}
    for tag, extra in (("plain", []), ("tuned", ["--autotune=1"])):
        env["OUT_DIR"] = str(tmp_path / tag) + "/"
        r = subprocess.run(["bash", str(run_dir / "main_recon_online_mirror_tile_vissfast.sh"), "--sky_gen=5", *extra],
                           cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        assert "exit code: 0" in r.stdout
        assert ("Autotune:" in r.stdout) == bool(extra)
        outs[tag] = np.fromfile(tmp_path / tag / "C1day1M.bin", dtype=np.float32)
        assert outs[tag].size == 12 * 32 * 32
    e = rel_err(outs["plain"], outs["tuned"])
    assert e[0] < 2e-6 and e[1] < 2e-6, e
    env["OUT_DIR"] = str(tmp_path / "root") + "/"
    env["B_MODE"] = "bin"
    r = subprocess.run(["bash", str(run_dir / "main_recon_online.sh"), "--sky_gen=5"], cwd=tmp_path,
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert (tmp_path / "root" / "C1day1M.txt").exists() and (tmp_path / "root" / "Viss1day1M.txt").exists()


def test_multi_day_running_sum_and_resume(gpu, vb, tmp_path):
    """--day_count > 1 reuses one run context (vb_pipeline_set_day); the
    --accum_file running sum equals the sum of the daily images and resumes
    from its file like the upstream accumulator daemon (viss_monitor.py)."""
    exe = BIN / "main_recon_online_mirror_tile_vissfast"
    sky = tmp_path / "sky"
    common = ["--btag=1M", "--nside=16", "--segs=2", "--blockage=1", "--occ_mode=2", f"--sky_dir={sky}", "--gpus=0",
              "--B_mode=bin", "--C_mode=bin", "--orbit_seed=42", "--sky_gen=3"]
    a, b, c = tmp_path / "a", tmp_path / "b", tmp_path / "c"
    r = run(exe, common + ["--day_start=1", "--day_count=3", f"--out_dir={a}/", f"--accum_file={a}/sum.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    daily = [np.fromfile(a / f"C{d}day1M.bin", dtype=np.float32) for d in (1, 2, 3)]
    acc = np.fromfile(a / "sum.bin", dtype=np.float32)
    ref = np.sum([d.astype(np.float64) for d in daily], axis=0)
    assert np.abs(acc - ref).max() <= 1e-6 * np.abs(ref).max()
    log = (a / "sum.bin.log").read_text().splitlines()
    assert len(log) == 3 and [ln.split(" | ")[1] for ln in log] == ["C1", "C2", "C3"]
    # a later day in its own process equals the same day of the multi-day run
    r = run(exe, common + ["--day_start=3", "--day_count=1", f"--out_dir={b}/"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(b / "C3day1M.bin", dtype=np.float32).view(np.uint32), daily[2].view(np.uint32))
    # resume: days 1-2, then day 3 from the saved sum, daily files not kept
    r = run(exe, common + ["--day_start=1", "--day_count=2", f"--out_dir={c}/", f"--accum_file={c}/sum.bin"], tmp_path)
    assert r.returncode == 0, r.stderr
    r = run(exe, common + ["--day_start=3", "--day_count=1", f"--out_dir={c}/", f"--accum_file={c}/sum.bin",
                           "--keep_daily=0"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Resuming running sum" in r.stdout
    assert not (c / "C3day1M.bin").exists()
    acc2 = np.fromfile(c / "sum.bin", dtype=np.float32)
    assert np.abs(acc2 - acc).max() <= 1e-6 * np.abs(ref).max()


def test_dropin_sky_slab_streaming(gpu, vb, tmp_path):
    """--slab_pix streams the sky through the device (vb_pipeline_run_host in
    slabs): same C as the resident run to summation rounding, and the running
    sum works across slabs."""
    exe = BIN / "main_recon_online_mirror_tile_vissfast"
    sky = tmp_path / "sky"
    common = ["--btag=1M", "--nside=16", "--segs=2", "--blockage=1", "--occ_mode=2", f"--sky_dir={sky}", "--gpus=0",
              "--B_mode=bin", "--C_mode=bin", "--orbit_seed=42", "--sky_gen=4", "--day_start=1", "--day_count=2"]
    a, b = tmp_path / "a", tmp_path / "b"
    r = run(exe, common + [f"--out_dir={a}/"], tmp_path)
    assert r.returncode == 0, r.stderr
    r = run(exe, common + [f"--out_dir={b}/", "--slab_pix=1024", f"--accum_file={b}/sum.bin", "--autotune=1"],
            tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Autotune skipped" in r.stdout
    for d in (1, 2):
        Ca = np.fromfile(a / f"C{d}day1M.bin", dtype=np.float32)
        Cb = np.fromfile(b / f"C{d}day1M.bin", dtype=np.float32)
        e = rel_err(Cb, Ca)
        assert e[0] < 1e-6 and e[1] < 1e-6, (d, e)
    acc = np.fromfile(b / "sum.bin", dtype=np.float32)
    ref = sum(np.fromfile(b / f"C{d}day1M.bin", dtype=np.float32).astype(np.float64) for d in (1, 2))
    assert np.abs(acc - ref).max() <= 1e-6 * np.abs(ref).max()


def test_dropin_30mhz_default_sky_streams_in_slabs(gpu, vb, tmp_path):
    """The upstream's 30 MHz runs use nside 16384 (3.2e9 pixels; its 30 MHz
    scripts pass --nside=16384, and --nside=0 picks it from --btag=30M,
    main_recon_online.cu:33-37), whose stage-1 records alone need ~150 GB: the
    drop-in finds that the resident sky does not fit and streams it in slabs
    by itself.  A short synthetic day (4 satellites x 16 steps) keeps it quick;
    C at 4096 sampled pixels equals the Python API's run with the same slabs."""
    exe = BIN / "main_recon_online_mirror_tile_vissfast"
    out = tmp_path / "out"
    args = ["--btag=30M", "--nside=16384", "--segs=2", "--blockage=1", "--occ_mode=2", f"--sky_dir={tmp_path}/sky", "--gpus=0",
            "--B_mode=bin", "--C_mode=bin", "--orbit_seed=42", "--sky_gen=5", "--orbit_model=synthetic", "--nsat=4",
            "--tsteps=16", "--occ_R_m=6371e3", "--grid_res=65", "--bl_max_m=0", f"--out_dir={out}/"]
    try:
        _check_30mhz_run(vb, exe, args, out, tmp_path)
    finally:                                  # the sky and C files are 12.9 GB each
        for f in (tmp_path / "sky" / "B_30M.bin", out / "C1day30M.bin"):
            f.unlink(missing_ok=True)


def _check_30mhz_run(vb, exe, args, out, tmp_path):
    import re
    r = run(exe, args, tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    m = re.search(r"streaming it in slabs of (\d+) pixels", r.stdout)
    assert m, r.stdout[-2000:]
    slab = int(m.group(1))
    npix = 12 * 16384 ** 2
    Cfile = out / "C1day30M.bin"
    assert Cfile.stat().st_size == 4 * npix
    idx = np.sort(np.random.default_rng(2).choice(npix, 4096, replace=False))
    Cd = np.memmap(Cfile, dtype=np.float32, mode="r")[idx].copy()
    assert np.isfinite(Cd).all() and np.abs(Cd).max() > 0
    B = vb.synthetic_sky(16384, seed=5)
    kw = dict(nside=16384, orbit_model=vb.ORBIT_SYNTHETIC, nsat=4, tsteps=16, segs=2, lambda_m=vb.btag_lambda("30M"),
              occ_R_m=6371e3, cull="tilecone", viss_tile_pix=256, mirror=1, grid_res=65, bl_max_m=0.0,
              occ_mode=2, blockage=1, orbit_seed=42, slab_pix=slab)
    with vb.Pipeline(vb.run_config(**kw)) as p:
        Cp, _, rep = p.run_host(B)
    assert rep["error_flags"] == 0
    e = rel_err(Cd, Cp[idx])
    assert e[0] < 1e-6 and e[1] < 1e-6, e
