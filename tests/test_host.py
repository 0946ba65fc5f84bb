"""The product's host-side preprocessing (liblab200.so, no GPU needed) is
bit-identical to the reference: level sets, RCM, IC(0), splits, transpose,
permute and CSR validation, checked against the golden fixtures and the
oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_matrices, strict_triangle


def test_topological_sort2_bit_exact(lab, golden):
    n_checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/topoL_levels" not in golden:
            continue
        for tag, lower in (("L", True), ("U", False)):
            t_ai, t_aj, _ = strict_triangle(n, ai, aj, av, lower)
            lv, ip, pf = lab.TopologicalSort2("L" if lower else "U", n, 0, t_ai, t_aj)
            assert lv == int(golden[f"{name}/topo{tag}_levels"][0]), name
            assert np.array_equal(ip, golden[f"{name}/topo{tag}_iperm"]), name
            assert np.array_equal(pf, golden[f"{name}/topo{tag}_prefix"]), name
            n_checked += 1
    assert n_checked >= 16


def test_topological_sort2_base1_and_large(lab, orc):
    from linearalgebra_b200 import gen
    P = orc.ptr
    n, ai, aj, av = gen.laplacian_3d(24)
    for lower in (True, False):
        t_ai, t_aj, _ = strict_triangle(n, ai, aj, av, lower)
        lv, ip, pf = lab.TopologicalSort2("L" if lower else "U", n, 0, t_ai, t_aj)
        ip2, pf2 = np.empty(n, np.int32), np.empty(n + 1, np.int32)
        lv2 = orc.port().oracle_topological_sort2(0 if lower else 1, n, 0, P(t_ai), P(t_aj), P(ip2), P(pf2))
        assert lv == lv2 == 3 * 23 + 1
        assert np.array_equal(ip, ip2) and np.array_equal(pf, pf2[: lv + 1])
        # one-based input gives the same levels with one-based iperm values
        lv1, ip1, pf1 = lab.TopologicalSort2("L" if lower else "U", n, 1, t_ai + 1, t_aj + 1)
        assert lv1 == lv and np.array_equal(ip1, ip + 1) and np.array_equal(pf1, pf)


def test_rcm_bit_exact(lab, golden, orc):
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/rcm_iperm" not in golden:
            continue
        ip, pm = lab.SerialCM(n, 0, ai, aj)
        assert np.array_equal(ip, golden[f"{name}/rcm_iperm"]), name
        assert np.array_equal(pm, golden[f"{name}/rcm_perm"]), name
        # base invariance (tests/reordering_test.cpp:266-332)
        ip1, pm1 = lab.SerialCM(n, 1, ai + 1, aj + 1)
        assert np.array_equal(ip1, ip + 1) and np.array_equal(pm1, pm + 1)
        checked += 1
    assert checked >= 5
    from linearalgebra_b200 import gen
    rf = orc.ref()
    for g in (20, 33):
        n, ai, aj, av = gen.laplacian_3d(g)
        ip, pm = lab.SerialCM(n, 0, ai, aj)
        ip2, pm2 = np.empty(n, np.int32), np.empty(n, np.int32)
        P = orc.ptr
        orc.port().oracle_rcm(n, 0, P(ai), P(aj), P(ip2), P(pm2))
        assert np.array_equal(ip, ip2) and np.array_equal(pm, pm2)
        if rf is not None:
            rf.la_ref_serial_cm(n, 0, P(ai), P(aj), P(ip2), P(pm2))
            assert np.array_equal(ip, ip2) and np.array_equal(pm, pm2)
        assert np.array_equal(np.sort(ip), np.arange(n))


def test_rcm_rejects_unsymmetric_pattern(lab, golden):
    ai, aj = golden["gd01c/ai"], golden["gd01c/aj"]
    with pytest.raises(lab.LAError) as e:
        lab.SerialCM(len(ai) - 1, 0, ai, aj)
    assert e.value.name == "LA_ERR_INVALID_ARG"


def test_icc0_bit_exact_and_breakdown(lab, golden):
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/icc0" not in golden:
            continue
        f = lab.ICCLevelNumeric0(n, 0, golden[f"{name}/u_ai"], golden[f"{name}/u_aj"],
                                 golden[f"{name}/u_av"])
        assert np.array_equal(f, golden[f"{name}/icc0"]), name
        checked += 1
    assert checked >= 4
    # ex5 breaks down without a shift (the reference returns false) ...
    from linearalgebra_b200 import gen
    ai, aj, av = golden["ex5/ai"], golden["ex5/aj"], golden["ex5/av"]
    n = len(ai) - 1
    ua, uj, uv = gen.upper_with_diag(n, ai, aj, av)
    with pytest.raises(lab.LAError) as e:
        lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    assert e.value.name == "LA_ERR_BREAKDOWN"
    # ... and the shift-retry loop (incomplete_cholesky.cpp:322-333) recovers
    f, shift = lab.ICCShifted(n, 0, ua, uj, uv)
    assert shift >= 1e-3 and np.all(np.isfinite(f))


def test_icc0_matches_oracle_on_mid_size(lab, orc):
    from linearalgebra_b200 import gen
    P = orc.ptr
    for n, ai, aj, av in (gen.stencil27(14, seed=3), gen.aniso7(14, seed=5)):
        ua, uj, uv = gen.upper_with_diag(n, ai, aj, av)
        f = lab.ICCLevelNumeric0(n, 0, ua, uj, uv, omega=0.25)
        f2 = np.empty_like(uv)
        assert orc.port().oracle_icc0(n, 0, P(ua), P(uj), P(uv), 0.25, P(f2)) == 1
        assert np.array_equal(f, f2)


def test_split_transpose_permute(lab, golden, orc):
    P = orc.ptr
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if m != n:
            continue
        (l_ai, l_aj, l_av), d, (u_ai, u_aj, u_av) = lab.SplitLDU(n, 0, ai, aj, av)
        assert np.array_equal(d, golden[f"{name}/ldu_D"])
        assert len(l_aj) == int(golden[f"{name}/ldu_Lnnz"][0])
        assert len(u_aj) == int(golden[f"{name}/ldu_Unnz"][0])
        e_ai, e_aj, e_av = strict_triangle(n, ai, aj, av, True)
        assert np.array_equal(l_ai, e_ai) and np.array_equal(l_aj, e_aj) and np.array_equal(l_av, e_av)
        t_ai, t_aj, t_av = lab.SplitTriangle("U", n, 0, ai, aj, av)
        o_ai, o_aj, o_av = (np.empty(n + 1, np.int32), np.empty(len(aj), np.int32), np.empty(len(aj)))
        k = orc.port().oracle_split_triangle(1, n, 0, P(ai), P(aj), P(av), P(o_ai), P(o_aj), P(o_av))
        assert np.array_equal(t_ai, o_ai) and np.array_equal(t_aj, o_aj[:k]) and np.array_equal(t_av, o_av[:k])
        # transpose twice is the identity (tests/uncatergorized_test.cpp:14-150)
        a1, j1, v1 = lab.Transpose(n, n, 0, ai, aj, av)
        a2, j2, v2 = lab.Transpose(n, n, 0, a1, j1, v1)
        assert np.array_equal(a2, ai) and np.array_equal(j2, aj) and np.array_equal(v2, av)
        rf = orc.ref()
        if rf is not None:
            r_ai, r_aj, r_av = np.empty(n + 1, np.int32), np.empty(len(aj), np.int32), np.empty(len(aj))
            rf.la_ref_transpose(n, n, 0, P(ai), P(aj), P(av), P(r_ai), P(r_aj), P(r_av))
            assert np.array_equal(a1, r_ai) and np.array_equal(j1, r_aj) and np.array_equal(v1, r_av)
        # symmetric permutation round trip (tests/mkl_sparse_mat_test.cpp:310-370)
        perm = np.random.default_rng(7).permutation(n).astype(np.int32)
        iperm = np.empty(n, np.int32)
        iperm[perm] = np.arange(n, dtype=np.int32)
        b_ai, b_aj, b_av = lab.Permute(n, 0, ai, aj, av, iperm, perm)
        c_ai, c_aj, c_av = lab.Permute(n, 0, b_ai, b_aj, b_av, perm, iperm)
        assert np.array_equal(c_ai, ai) and np.array_equal(c_aj, aj) and np.array_equal(c_av, av)
        if rf is not None:
            r_ai, r_aj, r_av = np.empty(n + 1, np.int32), np.empty(len(aj), np.int32), np.empty(len(aj))
            rf.la_ref_permute(n, 0, P(ai), P(aj), P(av), P(iperm), P(perm), P(r_ai), P(r_aj), P(r_av))
            assert np.array_equal(b_ai, r_ai) and np.array_equal(b_aj, r_aj) and np.array_equal(b_av, r_av)


def test_valid_csr_rejects_bad_input(lab):
    ai = np.array([0, 2, 3], np.int32)
    assert lab.ValidCSR(2, 2, 0, ai, np.array([0, 1, 1], np.int32))
    assert not lab.ValidCSR(2, 2, 0, ai, np.array([1, 0, 1], np.int32))   # unsorted
    assert not lab.ValidCSR(2, 2, 0, ai, np.array([1, 1, 1], np.int32))   # duplicate
    assert not lab.ValidCSR(2, 2, 0, ai, np.array([0, 1, 2], np.int32))   # out of range
    assert not lab.ValidCSR(2, 2, 1, ai, np.array([0, 1, 1], np.int32))   # ai[0] != base
    assert not lab.ValidCSR(2, 2, 0, np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32))
