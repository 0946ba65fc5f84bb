"""Pin the CPU oracle (oracle/la_oracle.c) before trusting it.

1. Against the committed golden fixtures (outputs of the reference's own
   code, tests/golden/make_golden.py): bit-exact for SpMV in all three forms
   at the reference's thread counts, level sets, RCM and IC(0).
2. Against the reference compiled in place (oracle/_ref), live, on seeded
   inputs the fixtures do not hold (skipped where it was not built).
3. Re-pins what the reference leaves unasserted (SegSum / ALBUS accuracy,
   tests/spmv_test.cpp:172-177, 209-214; IC values, precond_test.cpp:163-168).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_matrices, strict_triangle


def _spmv(orc, form, T, m, ai, aj, av, x, y0, a=1.5, b=0.5):
    po = orc.port()
    y = y0.copy()
    P = orc.ptr
    if form == "serial":
        po.oracle_serial_spmv(m, 0, P(ai), P(aj), P(av), P(x), P(y), a, b)
    else:
        getattr(po, f"oracle_{form}_spmv")(T, m, 0, P(ai), P(aj), P(av), P(x), P(y), a, b)
    return y


def test_oracle_spmv_matches_golden_bit_exact(orc, golden):
    for name, m, n, ai, aj, av in golden_matrices(golden):
        x, y0 = golden[f"{name}/spmv_x"], golden[f"{name}/spmv_y0"]
        assert np.array_equal(_spmv(orc, "serial", 0, m, ai, aj, av, x, y0),
                              golden[f"{name}/spmv_serial"]), name
        for T in (7, 10):
            for form in ("segsum", "albus"):
                got = _spmv(orc, form, T, m, ai, aj, av, x, y0)
                assert np.array_equal(got, golden[f"{name}/spmv_{form}_T{T}"]), (name, form, T)


def test_oracle_segsum_albus_accuracy_repinned(orc, golden):
    """The reference only prints these errors; pin them at 1e-14."""
    for name, m, n, ai, aj, av in golden_matrices(golden):
        x, y0 = golden[f"{name}/spmv_x"], golden[f"{name}/spmv_y0"]
        ref = golden[f"{name}/spmv_serial"]
        for T in (1, 3, 7, 10, 64):
            for form in ("segsum", "albus"):
                got = _spmv(orc, form, T, m, ai, aj, av, x, y0)
                err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
                assert err <= 1e-14, (name, form, T, err)


def test_oracle_topological_sort2_matches_golden(orc, golden):
    po = orc.port()
    P = orc.ptr
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/topoL_levels" not in golden:
            continue
        for tag, lower in (("L", True), ("U", False)):
            t_ai, t_aj, _ = strict_triangle(n, ai, aj, av, lower)
            ip = np.empty(n, np.int32)
            pf = np.empty(n + 1, np.int32)
            lv = po.oracle_topological_sort2(0 if lower else 1, n, 0, P(t_ai), P(t_aj), P(ip), P(pf))
            assert lv == int(golden[f"{name}/topo{tag}_levels"][0])
            assert np.array_equal(ip, golden[f"{name}/topo{tag}_iperm"])
            assert np.array_equal(pf[: lv + 1], golden[f"{name}/topo{tag}_prefix"])


def test_oracle_rcm_and_icc0_match_golden(orc, golden):
    po = orc.port()
    P = orc.ptr
    seen_rcm = seen_icc = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/rcm_iperm" in golden:
            ip, pm = np.empty(n, np.int32), np.empty(n, np.int32)
            po.oracle_rcm(n, 0, P(ai), P(aj), P(ip), P(pm))
            assert np.array_equal(ip, golden[f"{name}/rcm_iperm"]), name
            assert np.array_equal(pm, golden[f"{name}/rcm_perm"]), name
            seen_rcm += 1
        if f"{name}/icc0" in golden:
            ua, uj, uv = golden[f"{name}/u_ai"], golden[f"{name}/u_aj"], golden[f"{name}/u_av"]
            f = np.empty_like(uv)
            assert po.oracle_icc0(n, 0, P(ua), P(uj), P(uv), 0.0, P(f)) == 1
            assert np.array_equal(f, golden[f"{name}/icc0"]), name
            seen_icc += 1
    assert seen_rcm >= 5 and seen_icc >= 4


def test_oracle_triangular_solves_match_golden(orc, golden):
    po = orc.port()
    P = orc.ptr
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/fwd_unit" not in golden:
            continue
        l_ai, l_aj, l_av = strict_triangle(n, ai, aj, av, True)
        u_ai, u_aj, u_av = strict_triangle(n, ai, aj, av, False)
        b = np.ones(n)
        x = np.zeros(n)
        po.oracle_forward_substitution(n, 0, P(l_ai), P(l_aj), P(l_av), P(b), P(x))
        ref = golden[f"{name}/fwd_unit"]
        assert np.allclose(x, ref, rtol=1e-14, atol=0) or \
            np.linalg.norm(x - ref) <= 1e-14 * np.linalg.norm(ref), name
        if f"{name}/bwd_diag" in golden:
            d = golden[f"{name}/ldu_D"]
            po.oracle_backward_substitution(n, 0, P(u_ai), P(u_aj), P(u_av), P(d), P(b), P(x))
            ref = golden[f"{name}/bwd_diag"]
            assert np.linalg.norm(x - ref) <= 1e-14 * np.linalg.norm(ref), name


def test_oracle_vs_live_reference_seeded(orc):
    rf = orc.ref()
    if rf is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    from linearalgebra_b200 import gen
    P = orc.ptr
    po = orc.port()
    for seed in range(3):
        n, ai, aj, av = gen.powerlaw(5000 + 777 * seed, seed=seed, max_len=2500)
        x = np.random.default_rng(seed).uniform(-1, 1, n)
        y0 = np.random.default_rng(seed + 10).uniform(-1, 1, n)
        for T in (2, 5, 13):
            for form in ("segsum", "albus"):
                h = getattr(rf, f"la_ref_{form}_create")(T, n, 0, P(ai), P(aj), P(av))
                yr = y0.copy()
                getattr(rf, f"la_ref_{form}_apply")(h, n, 0, P(ai), P(aj), P(av), P(x), P(yr), -0.7, 1.25)
                getattr(rf, f"la_ref_{form}_destroy")(h)
                yo = _spmv(orc, form, T, n, ai, aj, av, x, y0, -0.7, 1.25)
                assert np.array_equal(yr, yo), (seed, T, form)
    # RCM + levels on a structurally symmetric 3D grid
    n, ai, aj, av = gen.laplacian_3d(12)
    ip1, pm1, ip2, pm2 = (np.empty(n, np.int32) for _ in range(4))
    rf.la_ref_serial_cm(n, 0, P(ai), P(aj), P(ip1), P(pm1))
    po.oracle_rcm(n, 0, P(ai), P(aj), P(ip2), P(pm2))
    assert np.array_equal(ip1, ip2) and np.array_equal(pm1, pm2)


def test_oracle_pcg_matches_reference_composed_pcg(orc, golden):
    rf = orc.ref()
    if rf is None:
        pytest.skip("oracle/_ref not built")
    P = orc.ptr
    po = orc.port()
    for name in ("lap2d_32", "lap3d_8", "st27_6", "aniso_6"):
        ai, aj, av = golden[f"{name}/ai"], golden[f"{name}/aj"], golden[f"{name}/av"]
        n = len(ai) - 1
        ua, uj, f = golden[f"{name}/u_ai"], golden[f"{name}/u_aj"], golden[f"{name}/icc0"]
        b = np.random.default_rng(0).uniform(-1, 1, n)
        x1, x2 = np.zeros(n), np.zeros(n)
        r1, r2 = np.zeros(1), np.zeros(1)
        h = rf.la_ref_pcg_create(2, n, 0, P(ai), P(aj), P(av), P(ua), P(uj), P(f))
        it1 = rf.la_ref_pcg_solve(h, P(b), P(x1), 1e-10, 5000, P(r1))
        rf.la_ref_pcg_destroy(h)
        it2 = po.oracle_pcg(n, 0, P(ai), P(aj), P(av), P(ua), P(uj), P(f), P(b), P(x2), 1e-10, 5000, P(r2))
        assert it1 > 0 and abs(it1 - it2) <= 1, (name, it1, it2)
        assert r1[0] < 1e-10 and r2[0] < 1e-10
        assert np.linalg.norm(x1 - x2) <= 1e-9 * np.linalg.norm(x1)


def _random_triangle(n, seed, lower, base):
    """Strict triangle with 0-6 entries per row, columns sorted, values in
    [-0.4, 0.4] (so unit solves stay bounded), indices carrying `base`."""
    r = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        pool = i if lower else n - 1 - i
        k = min(int(r.integers(0, 7)), pool)
        c = r.choice(pool, k, replace=False) if k else np.zeros(0, np.int64)
        rows.append(np.sort(c if lower else c + i + 1))
    ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32) + base
    aj = (np.concatenate(rows) if ai[-1] > base else np.zeros(0)).astype(np.int32) + base
    return ai, aj, r.uniform(-0.4, 0.4, int(ai[-1] - base))


def test_oracle_triangular_solves_match_live_reference(orc):
    """The oracle's restatements of the reference's triangular solves --
    ForwardSubstitution, BackwardSubstitution, ForwardSubstitutionT and the
    level-scheduled forms (triangle_solve.hpp:32-145) -- against the compiled
    reference on seeded random triangles, base 0 and 1, several thread
    counts for the level forms: bit for bit."""
    rf = orc.ref()
    if rf is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    P = orc.ptr
    po = orc.port()
    for seed, n in ((0, 1), (1, 37), (2, 2000), (3, 9000)):
        for base in (0, 1):
            b = np.random.default_rng(seed + 100).uniform(-1, 1, n)
            d = np.random.default_rng(seed + 200).uniform(1, 2, n)
            l_ai, l_aj, l_av = _random_triangle(n, seed, True, base)
            u_ai, u_aj, u_av = _random_triangle(n, seed + 50, False, base)
            x1, x2 = np.zeros(n), np.zeros(n)
            rf.la_ref_forward_substitution(n, base, P(l_ai), P(l_aj), P(l_av), P(b), P(x1))
            po.oracle_forward_substitution(n, base, P(l_ai), P(l_aj), P(l_av), P(b), P(x2))
            assert np.array_equal(x1, x2), (seed, base, "forward")
            rf.la_ref_backward_substitution(n, base, P(u_ai), P(u_aj), P(u_av), P(d), P(b),
                                            P(x1))
            po.oracle_backward_substitution(n, base, P(u_ai), P(u_aj), P(u_av), P(d), P(b),
                                            P(x2))
            assert np.array_equal(x1, x2), (seed, base, "backward")
            rf.la_ref_forward_substitution_t(n, base, P(u_ai), P(u_aj), P(u_av), P(b), P(x1))
            po.oracle_forward_substitution_t(n, base, P(u_ai), P(u_aj), P(u_av), P(b), P(x2))
            assert np.array_equal(x1, x2), (seed, base, "forward T")
            for uplo, (t_ai, t_aj, t_av), diag in ((0, (l_ai, l_aj, l_av), None),
                                                   (1, (u_ai, u_aj, u_av), d)):
                ip = np.empty(n, np.int32)
                pf = np.empty(n + 1, np.int32)
                lv = po.oracle_topological_sort2(uplo, n, base, P(t_ai), P(t_aj), P(ip), P(pf))
                po.oracle_level_solve(lv, P(ip), P(pf), base, P(t_ai), P(t_aj), P(t_av),
                                      P(diag), P(b), P(x2))
                for T in (1, 3, 8):
                    x1 = np.zeros(n)
                    if uplo == 0:
                        rf.la_ref_level_forward(T, P(ip), P(pf), lv, n, base, P(t_ai), P(t_aj),
                                                P(t_av), P(b), P(x1))
                    else:
                        rf.la_ref_level_backward(T, P(ip), P(pf), lv, n, base, P(t_ai), P(t_aj),
                                                 P(t_av), P(diag), P(b), P(x1))
                    assert np.array_equal(x1, x2), (seed, base, uplo, T, "level")
