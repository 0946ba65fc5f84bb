"""The C-ABI library loads and exports every entry point include/*.h
declares; device entry points fail loudly (no CPU fallback) without a GPU."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(la_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("la_csr_create", "la_spmv_plan_create", "la_spmv", "la_spmv_host",
                 "la_spmv_transpose", "la_sddmm_pattern", "la_trsv_analysis", "la_trsv",
                 "la_topological_sort2", "la_rcm", "la_icc0", "la_pcg_create", "la_pcg_solve",
                 "la_last_error_string"):
        assert must in names


def test_library_exports_every_declared_symbol(lab):
    so = ROOT / "linearalgebra_b200" / "liblab200.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (la_[a-z0-9_]+)\b", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    from linearalgebra_b200 import _lib
    assert set(_lib.exported_symbols()) <= exported


def test_version_and_error_string(lab):
    L = lab.lib()
    assert b"sm_100a" in L.la_version()
    assert isinstance(L.la_last_error_string(), bytes)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_device_entry_points_fail_loudly_without_gpu(lab):
    ai = np.array([0, 1], np.int32)
    aj = np.array([0], np.int32)
    av = np.array([2.0])
    with pytest.raises(lab.LAError) as e:
        lab.CSR(1, 1, 0, ai, aj, av)
    assert e.value.name == "LA_ERR_NO_DEVICE"
    sms = C.c_int()
    assert lab.lib().la_device_sm_count(C.byref(sms)) == 7


def test_invalid_csr_rejected_before_device(lab):
    with pytest.raises(lab.LAError) as e:
        lab.CSR(2, 2, 0, np.array([0, 2, 3], np.int32), np.array([1, 0, 1], np.int32),
                np.ones(3))
    assert e.value.name == "LA_ERR_BAD_CSR"


def test_transposed_solve_analysis_checks_before_device(lab):
    """la_trsv_analysis_transposed validates T's CSR on the host before it
    needs a GPU (unsorted columns -> LA_ERR_BAD_CSR); a strict upper triangle
    it accepts, and without a GPU it then fails loudly (LA_ERR_NO_DEVICE)."""
    ts = lab.OptimizedTriangularSolve("L")
    with pytest.raises(lab.LAError) as e:
        ts.analysis_transposed(3, 0, np.array([0, 2, 3, 3], np.int32),
                               np.array([2, 1, 2], np.int32), np.ones(3))
    assert e.value.name == "LA_ERR_BAD_CSR"
    # T upper -> T^T lower: an entry of T below its diagonal is not allowed
    with pytest.raises(lab.LAError) as e:
        ts.analysis_transposed(2, 0, np.array([0, 0, 1], np.int32),
                               np.array([0], np.int32), np.ones(1))
    assert e.value.name == "LA_ERR_INVALID_ARG"
    if not gpu_available():
        with pytest.raises(lab.LAError) as e:
            ts.analysis_transposed(3, 0, np.array([0, 2, 3, 3], np.int32),
                                   np.array([1, 2, 2], np.int32), np.ones(3))
        assert e.value.name == "LA_ERR_NO_DEVICE"
