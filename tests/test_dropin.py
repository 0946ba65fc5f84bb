"""The C++ drop-in layer (include/la_b200.hpp) compiled and run.

tests/dropin/dropin_main.cpp uses matrix_utils::b200 the way the
reference's callers use sparse_mat_op/ (SegSumSPMV, ALBUSSPMV, the SPMV<>
adapter over a CSRMatrix-like type, OptimizedTriangularSolve<FBST, L|U>,
the free solves, TopologicalSort2 / TopologicalSort, Diagonal, permute,
inversePermute).  It is compiled with g++ against the header and linked to
liblab200.so here; the host steps are checked on the CPU, the device classes
fail loudly without a GPU, and on a B200 their results are checked against
the reference's outputs frozen in tests/golden (signatures of
sparse_mat_op/spmv.hpp:310-334 and triangle_solve.hpp:149-208)."""
from __future__ import annotations

import shutil
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_matrices, gpu_available

SRC = ROOT / "tests" / "dropin" / "dropin_main.cpp"


@pytest.fixture(scope="module")
def dropin(lab, tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("dropin") / "dropin_main"
    libdir = ROOT / "linearalgebra_b200"
    subprocess.run([gxx, "-std=c++17", "-O1", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
                    str(SRC), f"-L{libdir}", "-llab200", f"-Wl,-rpath,{libdir}", "-o", str(out)],
                   check=True, capture_output=True, text=True)
    return out


def run(exe, tmp_path, n, ai, aj, av, x, y0, coo):
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(struct.pack("<ii", n, int(ai[-1])))
        for a, dt in ((ai, np.int32), (aj, np.int32), (av, np.float64), (x, np.float64),
                      (y0, np.float64)):
            f.write(np.ascontiguousarray(a, dt).tobytes())
    subprocess.run([str(exe), str(fin), str(fout), str(coo)], check=True, timeout=300)
    recs, buf, off = [], fout.read_bytes(), 0
    while off < len(buf):
        kind, count = struct.unpack_from("<iq", buf, off)
        off += 12
        dt, sz = (np.int32, 4) if kind == 0 else (np.float64, 8)
        recs.append(np.frombuffer(buf, dt, count, off).copy())
        off += sz * count
    return recs


def coo_file(golden, tmp_path, nm="K"):
    """One of the reference's own binary COO files (frozen bytes), base 1."""
    p = tmp_path / f"{nm}.bin"
    p.write_bytes(golden[f"bin_{nm}/bytes"].tobytes())
    return p


def cases(golden):
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if m == n and f"{name}/fwd_unit" in golden and f"{name}/bwd_diag" in golden:
            yield name, n, ai, aj, av, golden[f"{name}/spmv_x"], golden[f"{name}/spmv_y0"]


def test_dropin_host_steps(lab, dropin, golden, tmp_path):
    """Host functions through the C++ layer equal the reference's outputs;
    without a GPU the device classes throw LA_ERR_NO_DEVICE."""
    checked = 0
    coo = coo_file(golden, tmp_path)
    raw = np.frombuffer(coo.read_bytes(), np.dtype([("v", "<f8"), ("c", "<i4"), ("r", "<i4")]),
                        offset=8)
    for name, n, ai, aj, av, x, y0 in cases(golden):
        r = run(dropin, tmp_path, n, ai, aj, av, x, y0, coo)
        lv, ip, pf, last, kip, alld, diag, p_ai, p_aj, p_av, status = r[:11]
        cr, cc, cv, cmn = r[11:15]  # utils::b200::ReadFromBinaryCOO, host
        assert np.array_equal(cr, raw["r"]) and np.array_equal(cc, raw["c"])
        assert np.array_equal(cv, raw["v"])
        assert tuple(cmn) == tuple(golden["bin_K/base1_shape"])
        assert lv[0] == int(golden[f"{name}/topoL_levels"][0]), name
        assert np.array_equal(ip, golden[f"{name}/topoL_iperm"]), name
        assert np.array_equal(pf, golden[f"{name}/topoL_prefix"]), name
        assert np.array_equal(diag, golden[f"{name}/ldu_D"]), name
        rows = np.repeat(np.arange(n), np.diff(ai))
        assert alld[0] == int(np.all(np.bincount(rows[aj == rows], minlength=n) == 1)), name
        rev = np.arange(n, dtype=np.int32)[::-1].copy()
        want = lab.Permute(n, 0, ai, aj, av, rev, np.argsort(rev).astype(np.int32))
        assert all(np.array_equal(a, b) for a, b in zip((p_ai, p_aj, p_av), want)), name
        assert kip.size == n and np.array_equal(np.sort(kip), np.arange(n)), name
        if gpu_available():
            assert status[0] == -1
        else:
            assert status[0] == 7, status  # LA_ERR_NO_DEVICE
        checked += 1
    assert checked >= 5


@pytest.mark.gpu
def test_dropin_device_classes(lab, orc, dropin, golden, tmp_path):
    """SpMV (both forms and the SPMV<> adapter) and the triangular solves
    through the C++ layer: within 1e-13 of the reference's SerialSPMV and
    substitutions; the free functions bit for bit."""
    P = orc.ptr
    checked = 0
    coo = coo_file(golden, tmp_path)
    for name, n, ai, aj, av, x, y0 in cases(golden):
        r = run(dropin, tmp_path, n, ai, aj, av, x, y0, coo)
        assert r[10][0] == -1
        seg, alb, ad, lsol, usol, fwd, bwd, lfwd, lbwd, fwdt = r[15:25]
        bai, baj, bav, bmn = r[25:29]  # utils::b200::ReadFromBinaryCSR
        assert np.array_equal(bai, golden["bin_K/base1_ai"])
        assert np.array_equal(baj, golden["bin_K/base1_aj"])
        assert np.array_equal(bav, golden["bin_K/base1_av"])
        assert tuple(bmn) == tuple(golden["bin_K/base1_shape"])
        mai, maj, mav = r[29:32]  # utils::b200::read_matrix_market_csr
        assert np.array_equal(mai, ai) and np.array_equal(maj, aj), name
        assert np.array_equal(mav, av), name
        want = golden[f"{name}/spmv_serial"]
        for y in (seg, alb, ad):
            assert np.linalg.norm(y - want) <= 1e-13 * np.linalg.norm(want), name
        fu, bd = golden[f"{name}/fwd_unit"], golden[f"{name}/bwd_diag"]
        for got, want in ((lsol, fu), (fwd, fu), (lfwd, fu), (usol, bd), (bwd, bd), (lbwd, bd)):
            assert np.linalg.norm(got - want) <= 1e-13 * max(np.linalg.norm(want), 1e-300), name
        assert np.array_equal(fwd, fu, equal_nan=True), name
        assert np.array_equal(bwd, bd, equal_nan=True), name
        rows = np.repeat(np.arange(n), np.diff(ai))
        keep = aj > rows
        u_ai = np.zeros(n + 1, np.int32)
        np.cumsum(np.bincount(rows[keep], minlength=n), out=u_ai[1:])
        u_aj, u_av = np.ascontiguousarray(aj[keep], np.int32), np.ascontiguousarray(av[keep])
        ref = np.zeros(n)
        ones = np.ones(n)
        orc.port().oracle_forward_substitution_t(n, 0, P(u_ai), P(u_aj), P(u_av), P(ones), P(ref))
        assert np.linalg.norm(fwdt - ref) <= 1e-13 * max(np.linalg.norm(ref), 1e-300), name
        checked += 1
    assert checked >= 5
