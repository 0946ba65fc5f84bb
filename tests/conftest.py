"""Shared fixtures.  `-m gpu` tests need a B200; everything else runs on CPU.

The CUDA library and the oracle libraries are built in-tree on first use
(nvcc cross-compiles without a GPU)."""
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
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")


@pytest.fixture(scope="session")
def lab():
    from linearalgebra_b200 import build
    build.build()
    import linearalgebra_b200 as la
    la.lib()
    return la


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build(reference_too=True)
    return oracle


@pytest.fixture(scope="session")
def golden():
    """The committed fixtures (tests/golden/golden.npz) as a dict."""
    with np.load(GOLDEN / "golden.npz") as z:
        return {k: z[k] for k in z.files}


def golden_matrices(g):
    """Yield (name, m, n, ai, aj, av) for every matrix stored in the fixture."""
    names = sorted({k.split("/")[0] for k in g if k.endswith("/ai")})
    for name in names:
        ai, aj, av = g[f"{name}/ai"], g[f"{name}/aj"], g[f"{name}/av"]
        m, n = (int(v) for v in g[f"{name}/shape"])
        yield name, m, n, ai, aj, av


def strict_triangle(n, ai, aj, av, lower=True):
    rows = np.repeat(np.arange(n), np.diff(ai))
    keep = (aj < rows) if lower else (aj > rows)
    t_ai = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep], minlength=n), out=t_ai[1:])
    return t_ai, aj[keep].astype(np.int32), av[keep].astype(np.float64)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
