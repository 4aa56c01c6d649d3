"""The drop-in executables' text writers (viss_optimize_ws_b200/csrc/vb_text.h)
print exactly what the upstream iostream output prints: printf "%g" for C
and Viss, "%.15e" for the baseline tables (main_recon_online.cu:358-362,
516-538; common.hpp:145-153).  Built here with g++ against a tiny driver and
compared with Python's printf-style formatting (no GPU)."""
from __future__ import annotations

import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DRIVER = r'''
#include "vb_text.h"
#include <cstdio>
#include <vector>
int main(int argc, char** argv) {
  size_t n = 0;
  std::FILE* f = std::fopen(argv[1], "rb");
  std::fseek(f, 0, SEEK_END); n = std::ftell(f) / 4; std::fseek(f, 0, SEEK_SET);
  std::vector<float> v(n);
  if (std::fread(v.data(), 4, n, f) != n) return 2;
  std::fclose(f);
  // two columns interleaved (Viss layout), one column (C), three columns (baselines)
  bool ok = vbtext::write_rows(argv[2], {{v.data(), 2}, {v.data() + 1, 2}}, n / 2, vbtext::Fmt::General6);
  ok = ok && vbtext::write_rows(argv[3], {{v.data(), 1}}, n, vbtext::Fmt::General6);
  ok = ok && vbtext::write_rows(argv[4], {{v.data(), 3}, {v.data() + 1, 3}, {v.data() + 2, 3}}, n / 3,
                                vbtext::Fmt::Sci15);
  vbtext::AsyncWriter w(true);
  w.submit([&] { return vbtext::write_binary(argv[5], v.data(), n * 4); });
  ok = w.wait() && ok;
  return ok ? 0 : 1;
}
'''


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("vbtext")
    (d / "drv.cpp").write_text(DRIVER)
    exe = d / "drv"
    subprocess.run([gxx, "-O2", "-std=c++17", "-fopenmp", "-I", str(ROOT / "viss_optimize_ws_b200" / "csrc"),
                    str(d / "drv.cpp"), "-o", str(exe), "-pthread"], check=True, capture_output=True)
    return exe


def test_formats_match_printf(driver, tmp_path):
    rng = np.random.default_rng(4)
    special = np.array([0.0, -0.0, 1.0, -1.0, 0.1, 1e-30, -3.4e38, 3.4028235e38, 1.4e-45, -1.17549435e-38,
                        123456.7, 999999.5, 1e6, 1e-5, 1e-4, np.inf, -np.inf], np.float32)
    v = np.concatenate([special, (rng.standard_normal(200_001) * 10.0 ** rng.integers(-8, 8, 200_001))
                        .astype(np.float32)])
    v = v[: (v.size // 6) * 6]
    src = tmp_path / "v.bin"
    v.tofile(src)
    outs = [tmp_path / n for n in ("viss.txt", "c.txt", "uvw.txt", "c.bin")]
    subprocess.run([str(driver), str(src), *map(str, outs)], check=True)
    d = v.astype(np.float64)
    g = ["%g" % x for x in d]
    assert outs[0].read_text() == "".join(f"{g[i]} {g[i + 1]}\n" for i in range(0, d.size, 2))
    assert outs[1].read_text() == "".join(f"{x}\n" for x in g)
    e = ["%.15e" % x for x in d]
    assert outs[2].read_text() == "".join(f"{e[i]} {e[i + 1]} {e[i + 2]}\n" for i in range(0, d.size, 3))
    assert np.array_equal(np.fromfile(outs[3], np.float32).view(np.uint32), v.view(np.uint32))
