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


def test_split_transpose_large_threaded(lab, orc):
    """Above 2^18 entries the transpose, SplitLDU and SplitTriangle run on the
    host's threads: the same arrays as the one-pass restatements -- the
    compiled reference's transpose where available, scipy's otherwise, the
    oracle's SplitTriangle -- on a 27-point stencil (1.7M entries) and a
    random rectangular pattern with repeated-column-free ragged rows."""
    import scipy.sparse as sp
    from linearalgebra_b200 import gen
    P = orc.ptr
    n, ai, aj, av = gen.stencil27(40, seed=3)
    rng = np.random.default_rng(11)
    # ragged random rows (0 to 14 distinct sorted columns) over 70,000 columns
    lens = rng.integers(0, 15, 50_000)
    r_aj = np.concatenate([np.sort(rng.choice(70_000, k, replace=False)) for k in lens])
    r_ai = np.concatenate([[0], np.cumsum(lens)])
    cases = [(n, n, np.asarray(ai, np.int32), np.asarray(aj, np.int32), np.asarray(av)),
             (50_000, 70_000, r_ai.astype(np.int32), r_aj.astype(np.int32),
              rng.uniform(-1, 1, len(r_aj)))]
    for m, c, ai, aj, av in cases:
        assert ai[-1] >= (1 << 18)
        t_ai, t_aj, t_av = lab.Transpose(m, c, 0, ai, aj, av)
        T = sp.csr_matrix((av, aj, ai), shape=(m, c)).T.tocsr()
        T.sort_indices()
        assert np.array_equal(t_ai, T.indptr) and np.array_equal(t_aj, T.indices)
        assert np.array_equal(t_av, T.data)
        rf = orc.ref()
        if rf is not None and m == c:
            r_ai, r_aj, r_av = np.empty(m + 1, np.int32), np.empty(len(aj), np.int32), np.empty(len(aj))
            rf.la_ref_transpose(m, c, 0, P(ai), P(aj), P(av), P(r_ai), P(r_aj), P(r_av))
            assert np.array_equal(t_ai, r_ai) and np.array_equal(t_aj, r_aj)
            assert np.array_equal(t_av, r_av)
    # SplitLDU / SplitTriangle on the square case
    m, _, ai, aj, av = cases[0]
    (l_ai, l_aj, l_av), d, (u_ai, u_aj, u_av) = lab.SplitLDU(m, 0, ai, aj, av)
    for lower, (x_ai, x_aj, x_av) in ((True, (l_ai, l_aj, l_av)), (False, (u_ai, u_aj, u_av))):
        e_ai, e_aj, e_av = strict_triangle(m, ai, aj, av, lower)
        assert np.array_equal(x_ai, e_ai) and np.array_equal(x_aj, e_aj)
        assert np.array_equal(x_av, e_av)
    rows = np.repeat(np.arange(m), np.diff(ai))
    assert np.array_equal(d, av[aj == rows])
    for uplo, code in (("U", 1), ("L", 0)):
        t_ai, t_aj, t_av = lab.SplitTriangle(uplo, m, 0, ai, aj, av)
        o_ai, o_aj, o_av = (np.empty(m + 1, np.int32), np.empty(len(aj), np.int32), np.empty(len(aj)))
        k = orc.port().oracle_split_triangle(code, m, 0, P(ai), P(aj), P(av), P(o_ai), P(o_aj), P(o_av))
        assert np.array_equal(t_ai, o_ai) and np.array_equal(t_aj, o_aj[:k])
        assert np.array_equal(t_av, o_av[:k])


def test_valid_csr_rejects_bad_input(lab):
    ai = np.array([0, 2, 3], np.int32)
    assert lab.ValidCSR(2, 2, 0, ai, np.array([0, 1, 1], np.int32))
    assert not lab.ValidCSR(2, 2, 0, ai, np.array([1, 0, 1], np.int32))   # unsorted
    assert not lab.ValidCSR(2, 2, 0, ai, np.array([1, 1, 1], np.int32))   # duplicate
    assert not lab.ValidCSR(2, 2, 0, ai, np.array([0, 1, 2], np.int32))   # out of range
    assert not lab.ValidCSR(2, 2, 1, ai, np.array([0, 1, 1], np.int32))   # ai[0] != base
    assert not lab.ValidCSR(2, 2, 0, np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32))


def _strict(n, ai, aj, lower):
    rows = np.repeat(np.arange(n), np.diff(ai))
    keep = (aj < rows) if lower else (aj > rows)
    t_ai = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep], minlength=n), out=t_ai[1:])
    return t_ai, aj[keep].astype(np.int32)


def test_trsv_partition_never_reads_a_later_part(lab):
    """The partitioned solve's row partition (la_trsv_partition, host only):
    every part index in range, and no row reads a row of a higher-numbered
    part -- the property that makes the parts' dependency graph acyclic --
    for grids in natural and RCM order, both triangles, a 27-point stencil,
    random triangles with base 1, and 1, 3 or 148 parts.  A 7-point grid
    yields three cut coordinates and balanced parts; the 27-point stencil
    only the level (its documented limitation)."""
    from linearalgebra_b200 import gen
    cases = []
    n, ai, aj, av = gen.laplacian_3d(20)
    cases.append(("lap3d_20", n, ai, aj, 0, 3))
    iperm, perm = lab.SerialCM(n, 0, ai, aj)
    b_ai, b_aj, _ = lab.Permute(n, 0, ai, aj, av, iperm, perm)
    cases.append(("lap3d_20_rcm", n, b_ai, b_aj, 0, 3))
    n2, ai2, aj2, _ = gen.stencil27(10)
    cases.append(("st27_10", n2, ai2, aj2, 0, 1))
    n3, ai3, aj3, _ = gen.aniso7(14, seed=1)
    cases.append(("aniso7_14", n3, ai3, aj3, 0, None))
    rng = np.random.default_rng(7)
    m = 3000
    rows = [np.sort(rng.choice(m, min(m, 5), replace=False)) for _ in range(m)]
    r_ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    r_aj = np.concatenate(rows).astype(np.int32)
    cases.append(("random_base1", m, r_ai + 1, r_aj + 1, 1, None))
    for name, n, ai, aj, base, want_coords in cases:
        a0, j0 = (ai - base, aj - base)
        for lower in (True, False):
            t_ai, t_aj = _strict(n, a0, j0, lower)
            for nparts in (1, 3, 148):
                part, coords = lab.trsv_partition("L" if lower else "U", n, base,
                                                  t_ai + base, t_aj + base, nparts)
                assert part.shape == (n,) and part.min() >= 0 and part.max() < nparts, name
                r = np.repeat(np.arange(n), np.diff(t_ai))
                assert not np.any(part[t_aj] > part[r]), (name, lower, nparts)
                if nparts == 148 and want_coords is not None:
                    assert coords == want_coords, (name, lower, coords)
                if nparts == 148 and want_coords == 3:
                    sizes = np.bincount(part, minlength=nparts)
                    assert sizes.min() > 0 and sizes.max() <= 2 * n / nparts, (name, sizes.max())
    # the device form needs a GPU (without one: LA_ERR_NO_DEVICE, nothing computed)
    from conftest import gpu_available
    if not gpu_available():
        with pytest.raises(lab.LAError) as e:
            lab.trsv_partition("L", 1, 0, np.zeros(2, np.int32), np.zeros(0, np.int32), 4,
                               device=True)
        assert e.value.name == "LA_ERR_NO_DEVICE"
    # edge cases and argument checks
    assert lab.trsv_partition("L", 0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), 4)[0].size == 0
    part, _ = lab.trsv_partition("L", 1, 0, np.zeros(2, np.int32), np.zeros(0, np.int32), 4)
    assert part.tolist() == [0]
    with pytest.raises(lab.LAError) as e:
        lab.trsv_partition("L", 2, 0, np.array([0, 0, 1], np.int32), np.array([1], np.int32), 2)
    assert e.value.name == "LA_ERR_INVALID_ARG"


def test_topological_sort_kahn_bit_exact(lab, orc, golden):
    """TopologicalSort (matrix_utils.hpp:583-635, Kahn's order) against the
    compiled reference: iperm, prefix and the return value (the last level's
    index) bit for bit, both triangles, base 0 and 1, the golden matrices and
    seeded random triangles; the level sets equal TopologicalSort2's; a cycle
    is reported instead of looping."""
    rf = orc.ref()
    if rf is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    P = orc.ptr
    mats = [(name, n, ai, aj) for name, m, n, ai, aj, av in golden_matrices(golden) if m == n]
    rng = np.random.default_rng(11)
    for k, n in enumerate((1, 50, 3000)):
        rows = [np.sort(rng.choice(n, min(n, 4), replace=False)) for _ in range(n)]
        ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
        mats.append((f"random{k}", n, ai, np.concatenate(rows).astype(np.int32)))
    checked = 0
    for name, n, ai, aj in mats:
        for lower in (True, False):
            t_ai, t_aj, _ = strict_triangle(n, ai, aj, np.zeros(len(aj)), lower)
            for base in (0, 1):
                uplo = "L" if lower else "U"
                b_ai = np.ascontiguousarray(t_ai + base, np.int32)  # kept alive for the call
                b_aj = np.ascontiguousarray(t_aj + base, np.int32)
                r, ip, pf = lab.TopologicalSort(uplo, n, base, b_ai, b_aj)
                ip_ref = np.empty(n, np.int32)
                pf_ref = np.empty(n + 2, np.int32)
                r_ref = rf.la_ref_topological_sort(0 if lower else 1, n, base, P(b_ai), P(b_aj),
                                                   P(ip_ref), P(pf_ref))
                assert r == r_ref, (name, uplo, base)
                assert np.array_equal(ip, ip_ref), (name, uplo, base)
                assert np.array_equal(pf, pf_ref[: r_ref + 2]), (name, uplo, base)
                lv2, ip2, pf2 = lab.TopologicalSort2(uplo, n, base, b_ai, b_aj)
                assert lv2 == r + 1 and np.array_equal(pf, pf2), (name, uplo, base)
                for l in range(lv2):  # same rows per level, another order inside it
                    seg = slice(pf2[l], pf2[l + 1])
                    assert np.array_equal(np.sort(ip[seg]), np.sort(ip2[seg])), (name, l)
            checked += 1
    assert checked >= 10
    # n == 0, and a cycle (row 0 reads row 1, row 1 reads row 0)
    r, ip, pf = lab.TopologicalSort("L", 0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32))
    assert r == 0 and pf.tolist() == [0, 0]
    with pytest.raises(lab.LAError) as e:
        lab.TopologicalSort("L", 2, 0, np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    assert e.value.name == "LA_ERR_INVALID_ARG"


def test_permute_vec_inverse_permute_diagonal_bit_exact(lab, orc, golden):
    """permuteVec, inversePermute and Diagonal (matrix_utils.hpp:562-576,
    677-704; utils.cpp:101-108) against the compiled reference, base 0 and 1:
    bit for bit, Diagonal's bool included (the golden matrices without a full
    diagonal report false, the positions where the entry would go); rows only
    (permuteRow) is la_permute with no column permutation."""
    rf = orc.ref()
    if rf is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    P = orc.ptr
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if m != n:
            continue
        rng = np.random.default_rng(n)
        for base in (0, 1):
            perm = (rng.permutation(n) + base).astype(np.int32)
            ip = lab.InversePermute(perm, base)
            ip_ref = np.empty(n, np.int32)
            rf.la_ref_inverse_permute(n, base, P(perm), P(ip_ref))
            assert np.array_equal(ip, ip_ref), (name, base)
            v = rng.standard_normal(n)
            out_ref = np.empty(n)
            rf.la_ref_permute_vec(n, base, P(v), P(ip), P(out_ref))
            assert np.array_equal(lab.PermuteVec(n, base, v, ip), out_ref), (name, base)
            b_ai = np.ascontiguousarray(ai + base, np.int32)
            b_aj = np.ascontiguousarray(aj + base, np.int32)
            # the reference reads one value (and one column) past the row when
            # the last row lacks its diagonal: give it padded copies to read
            av_pad = np.append(av, 0.0)
            aj_pad = np.append(b_aj, np.int32(-1)).astype(np.int32)
            for invert in (False, True):
                ok, pos, d = lab.Diagonal(n, base, b_ai, b_aj, av, invert)
                pos_ref = np.empty(n, np.int32)
                d_ref = np.empty(n)
                ok_ref = rf.la_ref_diagonal(n, base, P(b_ai), P(aj_pad), P(av_pad), P(pos_ref),
                                            P(d_ref), int(invert))
                assert ok == bool(ok_ref), (name, base, invert)
                assert np.array_equal(pos, pos_ref), (name, base)
                full = np.ones(n, bool)
                if not ok:  # values past the last entry are undefined in the reference
                    full = pos - base < len(av)
                assert np.array_equal(d[full], d_ref[full]), (name, base, invert)
            # permuteRow: la_permute with rows only
            p_ai, p_aj, p_av = lab.Permute(n, base, b_ai, b_aj, av, ip, None)
            r_ai = np.empty(n + 1, np.int32)
            r_aj = np.empty(len(aj), np.int32)
            r_av = np.empty(len(aj))
            rf.la_ref_permute(n, base, P(b_ai), P(b_aj), P(av), P(ip), None, P(r_ai), P(r_aj),
                              P(r_av))
            assert np.array_equal(p_ai, r_ai) and np.array_equal(p_aj, r_aj), (name, base)
            assert np.array_equal(p_av, r_av), (name, base)
        checked += 1
    assert checked >= 5
    with pytest.raises(lab.LAError):
        lab.InversePermute(np.array([0, 0, 2], np.int32))


def _ilu0_python(n, ai, aj, av):
    """ILU(0), IKJ order, in plain Python (the same operations as la_ilu0)."""
    lu = av.astype(np.float64).copy()
    diag = [int(np.searchsorted(aj[ai[i]:ai[i + 1]], i)) + ai[i] for i in range(n)]
    for i in range(n):
        where = {int(aj[k]): k for k in range(ai[i], ai[i + 1])}
        for k in range(ai[i], diag[i]):
            c = int(aj[k])
            lu[k] = lu[k] / lu[diag[c]]
            for m in range(diag[c] + 1, ai[c + 1]):
                w = where.get(int(aj[m]))
                if w is not None:
                    lu[w] = lu[w] - lu[k] * lu[m]
    return lu


def test_ilu0_defining_property_and_restatement(lab):
    """la_ilu0: (L U)_ij = A_ij on A's pattern (L unit lower, U upper, both in
    A's pattern) to rounding, on stencils and a random diagonally dominant
    matrix; bit-identical to a plain-Python restatement; exact LU of a
    tridiagonal matrix; zero pivot and missing diagonal reported."""
    from linearalgebra_b200 import gen
    rng = np.random.default_rng(3)
    mats = [gen.laplacian_2d(12), gen.laplacian_3d(6), gen.stencil27(5)]
    m = 150
    dense = np.where(rng.random((m, m)) < 0.05, rng.uniform(-1, 1, (m, m)), 0.0)
    np.fill_diagonal(dense, np.abs(dense).sum(1) + 1.0)
    r, c = np.nonzero(dense)
    ai = np.concatenate([[0], np.cumsum(np.bincount(r, minlength=m))]).astype(np.int32)
    mats.append((m, ai, c.astype(np.int32), dense[r, c]))
    for n, ai, aj, av in mats:
        lu = lab.ILU0(n, 0, ai, aj, av)
        assert np.array_equal(lu, _ilu0_python(n, ai, aj, av))
        rows = np.repeat(np.arange(n), np.diff(ai))
        L = np.eye(n)
        U = np.zeros((n, n))
        low = aj < rows
        L[rows[low], aj[low]] = lu[low]
        U[rows[~low], aj[~low]] = lu[~low]
        A = np.zeros((n, n))
        A[rows, aj] = av
        prod = (L @ U)[rows, aj]
        assert np.max(np.abs(prod - av)) <= 1e-12 * np.max(np.abs(av)), n
    # tridiagonal: no fill, ILU(0) is the LU
    n = 40
    A = np.diag(np.full(n, 4.0)) + np.diag(np.full(n - 1, -1.0), 1) + np.diag(np.full(n - 1, -2.0), -1)
    r, c = np.nonzero(A)
    ai = np.concatenate([[0], np.cumsum(np.bincount(r, minlength=n))]).astype(np.int32)
    lu = lab.ILU0(n, 0, ai, c.astype(np.int32), A[r, c])
    L = np.eye(n)
    U = np.zeros((n, n))
    L[r[c < r], c[c < r]] = lu[c < r]
    U[r[c >= r], c[c >= r]] = lu[c >= r]
    assert np.allclose(L @ U, A, rtol=0, atol=1e-13)
    with pytest.raises(lab.LAError) as e:  # zero pivot in row 0
        lab.ILU0(2, 0, np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                 np.array([0.0, 1.0, 1.0, 1.0]))
    assert e.value.name == "LA_ERR_BREAKDOWN"
    with pytest.raises(lab.LAError) as e:  # row 1 has no diagonal
        lab.ILU0(2, 0, np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32),
                 np.array([1.0, 1.0]))
    assert e.value.name == "LA_ERR_INVALID_ARG"


def test_trsv_partition_large_nodes_thread_invariant():
    """A partition of over a million rows (the RCM-ordered 104^3 Laplacian's
    lower triangle, 1,124,864 rows, 128 parts), whose landmark searches,
    coordinate sums and k-d cuts run on the host's threads: the parts are the
    same at 1 and 8 threads, no row reads a later part, and the parts are
    balanced."""
    import os
    import subprocess
    import sys
    code = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import linearalgebra_b200 as la
from linearalgebra_b200 import gen
n, ai, aj, av = gen.laplacian_3d(104)
iperm, perm = la.SerialCM(n, 0, ai, aj)
b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
rows = np.repeat(np.arange(n), np.diff(b_ai))
keep = b_aj < rows
l_aj = b_aj[keep].astype(np.int32)
l_ai = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))]).astype(np.int32)
part, coords = la.trsv_partition("L", n, 0, l_ai, l_aj, 128)
np.savez(sys.argv[2], part=part, ai=l_ai, aj=l_aj, coords=coords)
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        got = []
        for t in ("1", "8"):
            out = os.path.join(d, f"p{t}.npz")
            env = dict(os.environ, OMP_NUM_THREADS=t)
            subprocess.run([sys.executable, "-c", code, root, out], check=True, env=env,
                           timeout=600)
            got.append(np.load(out))
        p1, p8 = got[0]["part"], got[1]["part"]
        assert np.array_equal(p1, p8)
        ai, aj = got[0]["ai"], got[0]["aj"]
        n = len(ai) - 1
        r = np.repeat(np.arange(n), np.diff(ai))
        assert not np.any(p1[aj] > p1[r])
        sizes = np.bincount(p1, minlength=128)
        assert int(got[0]["coords"]) == 3 and sizes.min() > 0 and sizes.max() <= 2 * n / 128
