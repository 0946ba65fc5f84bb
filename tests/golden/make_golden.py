"""Generate tests/golden/golden.npz from the reference itself.

Run in the container that holds the reference tree (it reads the
reference's own test matrices and calls the reference's own code compiled
in place as oracle/_ref/libla_ref.so):

    python tests/golden/make_golden.py

Stored per matrix <name>: the CSR (ai, aj, av, shape) and the reference's
outputs on it --
  spmv_x, spmv_y0                       seeded inputs (x ~ U[-1,1] seed 0,
                                        y0 ~ U[-1,1] seed 1)
  spmv_serial                           SerialSPMV, alpha 1.5, beta 0.5
  spmv_segsum_T{7,10}, spmv_albus_T{7,10}  SegSumSPMV / ALBUSSPMV with that
                                        many OpenMP threads, same alpha/beta
  spmv_ones                             SerialSPMV of ones, alpha 1, beta 0
                                        (tests/spmv_test.cpp:88-96)
and, for square matrices --
  topo{L,U}_levels/_iperm/_prefix       TopologicalSort2 on the strict
                                        triangles (matrix_utils.hpp:637-675)
  fwd_unit, bwd_diag                    OptimizedTriangularSolve<Barrier> (5
                                        threads, triangular_solve_test.cpp:208)
                                        on strict L (unit) and strict U with
                                        D from SplitLDU, b = ones
  rcm_iperm, rcm_perm                   SerialCM, structurally symmetric only
  icc0 (+ u_ai/u_aj/u_av)               ICCLevelNumeric IC(0) factor, SPD only
The matrices are the reference's test fixtures (tests/data/ex5.mtx,
rdist1.mtx, jgl009.mtx, data/GD01_c.mtx) and small seeded synthetic ones
from linearalgebra_b200.gen.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import ptr  # noqa: E402
from linearalgebra_b200 import gen, mmio  # noqa: E402

REF = oracle.reference_tree()
OUT = Path(__file__).resolve().parent / "golden.npz"


def strict(n, ai, aj, av, lower):
    rows = np.repeat(np.arange(n), np.diff(ai))
    keep = (aj < rows) if lower else (aj > rows)
    t_ai = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep], minlength=n), out=t_ai[1:])
    return t_ai, np.ascontiguousarray(aj[keep], np.int32), np.ascontiguousarray(av[keep])


def structurally_symmetric(n, ai, aj):
    rows = np.repeat(np.arange(n), np.diff(ai))
    a = set(zip(rows.tolist(), aj.tolist()))
    return all((c, r) in a for r, c in a)


def main():
    oracle.build(reference_too=True)
    rf = oracle.ref()
    assert rf is not None, "oracle/_ref was not built"
    mats = {}
    for nm, p in [("ex5", "tests/data/ex5.mtx"), ("rdist1", "tests/data/rdist1.mtx"),
                  ("jgl009", "tests/data/jgl009.mtx"), ("gd01c", "data/GD01_c.mtx")]:
        m, n, ai, aj, av = mmio.read_mtx(REF / p)
        mats[nm] = (m, n, ai, aj, av, False)
    for nm, t in [("lap2d_32", gen.laplacian_2d(32)), ("lap3d_8", gen.laplacian_3d(8)),
                  ("st27_6", gen.stencil27(6)), ("aniso_6", gen.aniso7(6)),
                  ("powerlaw_3000", gen.powerlaw(3000, max_len=1500))]:
        n, ai, aj, av = t
        mats[nm] = (n, n, ai, aj, av, nm != "powerlaw_3000")
    out = {}
    for nm, (m, n, ai, aj, av, spd) in mats.items():
        ai, aj, av = (np.ascontiguousarray(ai, np.int32), np.ascontiguousarray(aj, np.int32),
                      np.ascontiguousarray(av, np.float64))
        out[f"{nm}/ai"], out[f"{nm}/aj"], out[f"{nm}/av"] = ai, aj, av
        out[f"{nm}/shape"] = np.array([m, n])
        x = np.random.default_rng(0).uniform(-1, 1, n)
        y0 = np.random.default_rng(1).uniform(-1, 1, m)
        out[f"{nm}/spmv_x"], out[f"{nm}/spmv_y0"] = x, y0
        y = y0.copy()
        rf.la_ref_serial_spmv(m, 0, ptr(ai), ptr(aj), ptr(av), ptr(x), ptr(y), 1.5, 0.5)
        out[f"{nm}/spmv_serial"] = y
        for T in (7, 10):
            for form in ("segsum", "albus"):
                h = getattr(rf, f"la_ref_{form}_create")(T, m, 0, ptr(ai), ptr(aj), ptr(av))
                y = y0.copy()
                getattr(rf, f"la_ref_{form}_apply")(h, m, 0, ptr(ai), ptr(aj), ptr(av),
                                                     ptr(x), ptr(y), 1.5, 0.5)
                getattr(rf, f"la_ref_{form}_destroy")(h)
                out[f"{nm}/spmv_{form}_T{T}"] = y
        ones = np.ones(n)
        y = np.zeros(m)
        rf.la_ref_serial_spmv(m, 0, ptr(ai), ptr(aj), ptr(av), ptr(ones), ptr(y), 1.0, 0.0)
        out[f"{nm}/spmv_ones"] = y
        if m != n:
            continue
        for tag, lower in (("L", True), ("U", False)):
            t_ai, t_aj, _ = strict(n, ai, aj, av, lower)
            ip = np.empty(n, np.int32)
            pf = np.empty(n + 1, np.int32)
            lv = rf.la_ref_topological_sort2(0 if lower else 1, n, 0, ptr(t_ai), ptr(t_aj),
                                             ptr(ip), ptr(pf))
            out[f"{nm}/topo{tag}_levels"] = np.array([lv])
            out[f"{nm}/topo{tag}_iperm"] = ip
            out[f"{nm}/topo{tag}_prefix"] = pf[: lv + 1].copy()
        # triangular solves on SplitLDU pieces, b = ones
        nnz = len(aj)
        l_ai, u_ai = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
        l_aj, u_aj = np.empty(max(nnz, 1), np.int32), np.empty(max(nnz, 1), np.int32)
        l_av, u_av = np.empty(max(nnz, 1)), np.empty(max(nnz, 1))
        d = np.empty(n)
        ln, un = np.zeros(1, np.int32), np.zeros(1, np.int32)
        rf.la_ref_split_ldu(n, 0, ptr(ai), ptr(aj), ptr(av), ptr(l_ai), ptr(l_aj), ptr(l_av),
                            ptr(d), ptr(u_ai), ptr(u_aj), ptr(u_av), ptr(ln), ptr(un))
        out[f"{nm}/ldu_D"] = d.copy()
        out[f"{nm}/ldu_Lnnz"], out[f"{nm}/ldu_Unnz"] = ln.copy(), un.copy()
        b = np.ones(n)
        xs = np.zeros(n)
        h = rf.la_ref_trsv_create(0, 0, 5, n, 0, ptr(l_ai), ptr(l_aj), ptr(l_av), None)
        rf.la_ref_trsv_apply(h, ptr(b), ptr(xs))
        rf.la_ref_trsv_destroy(h)
        out[f"{nm}/fwd_unit"] = xs.copy()
        if np.all(d != 0):
            dd = d.copy()
            h = rf.la_ref_trsv_create(0, 1, 5, n, 0, ptr(u_ai), ptr(u_aj), ptr(u_av), ptr(dd))
            rf.la_ref_trsv_apply(h, ptr(b), ptr(xs))
            rf.la_ref_trsv_destroy(h)
            out[f"{nm}/bwd_diag"] = xs.copy()
        if structurally_symmetric(n, ai, aj):
            ip, pm = np.empty(n, np.int32), np.empty(n, np.int32)
            rf.la_ref_serial_cm(n, 0, ptr(ai), ptr(aj), ptr(ip), ptr(pm))
            out[f"{nm}/rcm_iperm"], out[f"{nm}/rcm_perm"] = ip, pm
        if spd:
            ua, uj, uv = gen.upper_with_diag(n, ai, aj, av)
            ua, uj, uv = (np.ascontiguousarray(ua, np.int32), np.ascontiguousarray(uj, np.int32),
                          np.ascontiguousarray(uv))
            f = np.empty_like(uv)
            ok = rf.la_ref_icc0(n, 0, ptr(ua), ptr(uj), ptr(uv), 0.0, ptr(f))
            assert ok
            out[f"{nm}/u_ai"], out[f"{nm}/u_aj"], out[f"{nm}/u_av"] = ua, uj, uv
            out[f"{nm}/icc0"] = f
    # binary COO ingest: the reference's own data/shared/*.bin files (raw
    # bytes) and what its ReadFromBinaryCSR (utils/utils.h:46-91) builds from
    # them, with the files' base 1 and read as base 0
    for nm in ("K", "M", "G", "G2"):
        path = REF / "data" / "shared" / f"{nm}.bin"
        out[f"bin_{nm}/bytes"] = np.frombuffer(path.read_bytes(), np.uint8).copy()
        for base in (1, 0):
            m, n = np.zeros(1, np.int32), np.zeros(1, np.int32)
            cnt = rf.la_ref_read_binary_csr(str(path).encode(), base, None, None, None,
                                            ptr(m), ptr(n))
            ai = np.zeros(int(m[0]) + 1, np.int32)
            aj = np.zeros(cnt, np.int32)
            av = np.zeros(cnt)
            rf.la_ref_read_binary_csr(str(path).encode(), base, ptr(ai), ptr(aj), ptr(av),
                                      ptr(m), ptr(n))
            key = f"bin_{nm}/base{base}"
            out[f"{key}_ai"], out[f"{key}_aj"], out[f"{key}_av"] = ai, aj, av
            out[f"{key}_shape"] = np.array([int(m[0]), int(n[0])])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
