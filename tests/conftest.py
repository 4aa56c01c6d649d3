"""Shared test fixtures.

Markers: `gpu` -- needs a CUDA device (run with -m gpu on the B200 box).
CPU tests (-m "not gpu") cover the oracle against the golden fixtures, host
logic, and that the C ABI library loads and exports every declared symbol.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def vb():
    """The product package with its CUDA library loaded (fails loudly if unbuilt)."""
    import viss_optimize_ws_b200 as vb
    vb.lib()
    return vb


@pytest.fixture(scope="session")
def gpu(vb):
    """A usable CUDA device; GPU tests fail (not skip) when the library is missing."""
    import ctypes as C
    sm, ma, mi = C.c_int(), C.c_int(), C.c_int()
    rc = vb.lib().vb_device_info(C.byref(sm), C.byref(ma), C.byref(mi))
    if rc != 0:
        pytest.skip("no CUDA device: " + vb.lib().vb_last_error().decode())
    return {"sms": sm.value, "cc": (ma.value, mi.value)}


@pytest.fixture(scope="session")
def orc():
    from oracle import py as orp
    orp.oracle()
    return orp


@pytest.fixture(scope="session")
def ref(orc):
    if not orc.ref_available():
        pytest.fail("upstream reference harness (oracle/_ref) is not built: run `make -C oracle ref`")
    return orc


def load_golden(name: str) -> dict:
    p = GOLDEN / f"{name}.npz"
    if not p.exists():
        pytest.skip(f"golden fixture {p.name} not present")
    with np.load(p, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def rel_err(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    """Normwise errors of a against reference b: (max|a-b| / max|b|, ||a-b||_2 / ||b||_2)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = a - b
    mb = np.max(np.abs(b)) if b.size else 0.0
    nb = np.linalg.norm(b)
    return (float(np.max(np.abs(d)) / mb) if mb > 0 else float(np.max(np.abs(d), initial=0.0)),
            float(np.linalg.norm(d) / nb) if nb > 0 else float(np.linalg.norm(d)))
