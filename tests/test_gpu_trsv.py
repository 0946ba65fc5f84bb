"""GPU level-scheduled triangular solves vs the oracle and the reference.

Level sets must match TopologicalSort2 bit-exactly; FP64 solutions agree
with the reference's OptimizedTriangularSolve<Barrier> to <= 1e-13
relative 2-norm; the FP32 plan states its error against the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_matrices, strict_triangle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
TOL = 1e-13


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dtype)


def solve(lab, uplo, n, t_ai, t_aj, t_av, diag, b, dtype=np.float64):
    ts = lab.OptimizedTriangularSolve(uplo, 5, dtype=dtype).analysis(n, 0, t_ai, t_aj, t_av, diag)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    x = torch.empty(n, dtype=tdt, device="cuda")
    ts(dev(b, tdt), x)
    return ts, x.double().cpu().numpy()


def test_trsv_golden_and_levels(lab, golden):
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if f"{name}/fwd_unit" not in golden:
            continue
        l_ai, l_aj, l_av = strict_triangle(n, ai, aj, av, True)
        ts, x = solve(lab, "L", n, l_ai, l_aj, l_av, None, np.ones(n))
        assert rel(x, golden[f"{name}/fwd_unit"]) <= TOL, name
        lv, ip, pf = ts.levels()
        assert lv == int(golden[f"{name}/topoL_levels"][0])
        assert np.array_equal(ip, golden[f"{name}/topoL_iperm"])
        assert np.array_equal(pf, golden[f"{name}/topoL_prefix"])
        if f"{name}/bwd_diag" in golden:
            u_ai, u_aj, u_av = strict_triangle(n, ai, aj, av, False)
            ts, x = solve(lab, "U", n, u_ai, u_aj, u_av, golden[f"{name}/ldu_D"], np.ones(n))
            assert rel(x, golden[f"{name}/bwd_diag"]) <= TOL, name
            lv, ip, pf = ts.levels()
            assert np.array_equal(ip, golden[f"{name}/topoU_iperm"])
        checked += 1
    assert checked >= 8


def _ic_factor_rcm(lab, n, ai, aj, av):
    """RCM-permute, IC(0)-factor; returns B (permuted A) and strict L=U^T,
    strict U, diag as the PCG preconditioner uses them."""
    from linearalgebra_b200 import gen
    iperm, perm = lab.SerialCM(n, 0, ai, aj)
    b_ai, b_aj, b_av = lab.Permute(n, 0, ai, aj, av, iperm, perm)
    ua, uj, uv = gen.upper_with_diag(n, b_ai, b_aj, b_av)
    f = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    _, d, (s_ai, s_aj, s_av) = lab.SplitLDU(n, 0, ua, uj, f)
    t_ai, t_aj, t_av = lab.Transpose(n, n, 0, s_ai, s_aj, s_av)
    return (b_ai, b_aj, b_av), (t_ai, t_aj, t_av), (s_ai, s_aj, s_av), d


def test_trsv_ic_factors_rcm(lab, orc):
    from linearalgebra_b200 import gen
    P = orc.ptr
    for n, ai, aj, av in (gen.laplacian_3d(32), gen.stencil27(20), gen.aniso7(24, seed=1)):
        _, (t_ai, t_aj, t_av), (s_ai, s_aj, s_av), d = _ic_factor_rcm(lab, n, ai, aj, av)
        b = np.random.default_rng(0).uniform(-1, 1, n)
        for uplo, (c_ai, c_aj, c_av) in (("L", (t_ai, t_aj, t_av)), ("U", (s_ai, s_aj, s_av))):
            ts, x = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b)
            lv, ip, pf = ts.levels()
            ref = np.zeros(n)
            orc.port().oracle_level_solve(lv, P(ip), P(pf), 0, P(c_ai), P(c_aj), P(c_av), P(d),
                                          P(b), P(ref))
            assert rel(x, ref) <= TOL, (n, uplo, rel(x, ref))
            # exact operations in the reference's in-row order: bit-identical
            assert np.array_equal(x, ref), (n, uplo, np.abs(x - ref).max())
            if uplo == "L":
                ser = np.zeros(n)
                orc.port().oracle_forward_substitution_diag(n, 0, P(c_ai), P(c_aj), P(c_av), P(d),
                                                            P(b), P(ser))
            else:
                ser = np.zeros(n)
                orc.port().oracle_backward_substitution(n, 0, P(c_ai), P(c_aj), P(c_av), P(d),
                                                        P(b), P(ser))
            assert rel(x, ser) <= TOL
            _, x32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
            e32 = rel(x32, ref)
            print(f"n={n} {uplo}: fp64 err {rel(x, ref):.2e}, fp32 err {e32:.2e}, levels {lv}")
            assert e32 <= 1e-4


def test_trsv_repeated_and_reference_levels_3d(lab, orc):
    """128^3 Laplacian under RCM keeps 3(g-1)+1 = 382 levels; repeated solves
    are identical (tests/triangular_solve_test.cpp repeats 100 times)."""
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_3d(128)
    _, (t_ai, t_aj, t_av), _, d = _ic_factor_rcm(lab, n, ai, aj, av)
    ts = lab.OptimizedTriangularSolve("L").analysis(n, 0, t_ai, t_aj, t_av, d)
    lv, ip, pf = ts.levels()
    assert lv == 382
    rf = orc.ref()
    if rf is not None:
        P = orc.ptr
        ip2, pf2 = np.empty(n, np.int32), np.empty(n + 1, np.int32)
        assert rf.la_ref_topological_sort2(0, n, 0, P(t_ai), P(t_aj), P(ip2), P(pf2)) == 382
        assert np.array_equal(ip, ip2) and np.array_equal(pf, pf2[:383])
    b = dev(np.random.default_rng(5).uniform(-1, 1, n))
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    ts(b, x)
    first = x.clone()
    for _ in range(100):
        ts(b, x)
    assert torch.equal(first, x)
    ref = np.zeros(n)
    P = orc.ptr
    bn = b.cpu().numpy()  # keep the host copy alive across the call
    orc.port().oracle_level_solve(lv, P(ip), P(pf), 0, P(t_ai), P(t_aj), P(t_av), P(d),
                                  P(bn), P(ref))
    assert np.array_equal(x.cpu().numpy(), ref)


def test_trsv_host_path(lab, golden):
    ai, aj, av = golden["lap2d_32/ai"], golden["lap2d_32/aj"], golden["lap2d_32/av"]
    n = len(ai) - 1
    l_ai, l_aj, l_av = strict_triangle(n, ai, aj, av, True)
    ts = lab.OptimizedTriangularSolve("L").analysis(n, 0, l_ai, l_aj, l_av)
    x = np.zeros(n)
    ts(np.ones(n), x)
    assert rel(x, golden["lap2d_32/fwd_unit"]) <= TOL


def _chain(n):
    """Row i reads row i - 1 (strict lower bidiagonal, values 0.5)."""
    ai = np.zeros(n + 1, np.int32)
    ai[2:] = np.arange(1, n, dtype=np.int32)
    return ai, np.arange(n - 1, dtype=np.int32), np.full(n - 1, 0.5)


def test_trsv_bounded_wait_reports_timeout(lab, orc):
    """A caller-built level set that schedules every row before the row it
    reads stalls the persistent solve (all resident warps wait on chunks no
    warp can claim).  The bounded waits end it with LA_ERR_TIMEOUT after about
    a second, without a fault, trap or hang, and the context stays usable."""
    import time
    n = 200_000
    ai, aj, av = _chain(n)
    iperm = np.arange(n, dtype=np.int32)[::-1].copy()
    prefix = np.array([0, n], np.int32)
    bad = lab.OptimizedTriangularSolve("L").analysis_levels(n, 0, ai, aj, av, iperm, prefix)
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    t0 = time.time()
    with pytest.raises(lab.LAError) as e:
        bad(b, x)
    assert e.value.name == "LA_ERR_TIMEOUT"
    assert time.time() - t0 < 30
    good = lab.OptimizedTriangularSolve("L").analysis(n, 0, ai, aj, av)
    good(b, x)
    ref = np.zeros(n)
    P = orc.ptr
    bn = np.ones(n)
    orc.port().oracle_forward_substitution(n, 0, P(ai), P(aj), P(av), P(bn), P(ref))
    assert np.array_equal(x.cpu().numpy(), ref)
    # a level order that respects the dependencies works through the same entry
    ok = lab.OptimizedTriangularSolve("L").analysis_levels(
        n, 0, ai, aj, av, np.arange(n, dtype=np.int32), np.arange(n + 1, dtype=np.int32))
    ok(b, x)
    assert np.array_equal(x.cpu().numpy(), ref)


def test_trsv_partitioned_bounded_wait_reports_timeout(lab, orc, monkeypatch):
    """The partitioned schedule's abort path: with LA_TRSV_STALL_TEST one row
    waits for its own, never published value, so its wait runs out after the
    1 s bound; every thread of every part leaves (the CTA-wide abort vote),
    the solve returns LA_ERR_TIMEOUT without a fault or hang, and the next
    plan on the same context solves correctly."""
    import time
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_3d(24)
    _, (t_ai, t_aj, t_av), _, d = _ic_factor_rcm(lab, n, ai, aj, av)
    b = torch.as_tensor(np.random.default_rng(4).uniform(-1, 1, n)).cuda()
    x = torch.empty_like(b)
    monkeypatch.setenv("LA_TRSV_SCHEDULE", "parts")
    for dt in (np.float64, np.float32):
        monkeypatch.setenv("LA_TRSV_STALL_TEST", "1")
        bad = lab.OptimizedTriangularSolve("L", dtype=dt).analysis(n, 0, t_ai, t_aj, t_av, d)
        assert bad.schedule()[0] == "parts"
        bb = b.to(torch.float64 if dt == np.float64 else torch.float32)
        xx = torch.empty_like(bb)
        t0 = time.time()
        with pytest.raises(lab.LAError) as e:
            bad(bb, xx)
        assert e.value.name == "LA_ERR_TIMEOUT"
        assert time.time() - t0 < 30
        monkeypatch.delenv("LA_TRSV_STALL_TEST")
    good = lab.OptimizedTriangularSolve("L").analysis(n, 0, t_ai, t_aj, t_av, d)
    good(b, x)
    lv, ip, pf = good.levels()
    ref = np.zeros(n)
    P = orc.ptr
    bn = b.cpu().numpy()
    orc.port().oracle_level_solve(lv, P(ip), P(pf), 0, P(t_ai), P(t_aj), P(t_av), P(d),
                                  P(bn), P(ref))
    assert np.array_equal(x.cpu().numpy(), ref)


def test_trsv_levels_validation(lab):
    ai, aj, av = _chain(8)
    with pytest.raises(lab.LAError):  # not a permutation
        lab.OptimizedTriangularSolve("L").analysis_levels(
            8, 0, ai, aj, av, np.zeros(8, np.int32), np.array([0, 8], np.int32))
    with pytest.raises(lab.LAError):  # prefix does not end at n
        lab.OptimizedTriangularSolve("L").analysis_levels(
            8, 0, ai, aj, av, np.arange(8, dtype=np.int32), np.array([0, 7], np.int32))


def _long_rows_lower(n, seed):
    """Strict lower triangle with a few rows longer than 16 entries (the
    partitioned schedule's CSR tail) and some empty rows."""
    r = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = 0 if i % 7 == 3 else (int(r.integers(17, 40)) if i % 97 == 50 else int(r.integers(0, 5)))
        k = min(k, i)
        rows.append(np.sort(r.choice(i, k, replace=False)) if k else np.zeros(0, np.int64))
    ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    aj = (np.concatenate(rows) if ai[-1] else np.zeros(0)).astype(np.int32)
    return ai, aj, r.uniform(-0.3, 0.3, int(ai[-1]))


@pytest.mark.parametrize("schedule", ["parts", "flags"])
def test_trsv_schedules_bit_identical(lab, orc, monkeypatch, schedule):
    """Both schedules -- level order with per-row readiness, and the
    partitioned one (co-resident CTAs, part values in shared memory) --
    give the oracle's level solve bit for bit, in both triangles and both
    storage precisions, including rows longer than the register slots and a
    forced small part count (many cross-part waits)."""
    from linearalgebra_b200 import gen
    P = orc.ptr
    monkeypatch.setenv("LA_TRSV_SCHEDULE", schedule)
    cases = []
    for n, ai, aj, av in (gen.laplacian_3d(40), gen.stencil27(16), gen.aniso7(28, seed=3)):
        _, lt, ut, d = _ic_factor_rcm(lab, n, ai, aj, av)
        cases += [(n, "L", lt, d), (n, "U", ut, d)]
    n = 30_000
    cases.append((n, "L", _long_rows_lower(n, 1), np.random.default_rng(2).uniform(1, 2, n)))
    for parts in (None, "3"):
        if parts:
            monkeypatch.setenv("LA_TRSV_PARTS", parts)
        for n, uplo, (c_ai, c_aj, c_av), d in cases:
            b = np.random.default_rng(n).uniform(-1, 1, n)
            ts, x = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b)
            assert ts.schedule()[0] == ("parts" if schedule == "parts" else "levels")
            lv, ip, pf = ts.levels()
            ref = np.zeros(n)
            orc.port().oracle_level_solve(lv, P(ip), P(pf), 0, P(c_ai), P(c_aj), P(c_av),
                                          P(d), P(b), P(ref))
            assert np.array_equal(x, ref), (n, uplo, schedule, parts)
            ts32, x32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
            assert rel(x32, ref) <= 1e-4
            # FP32 storage and arithmetic in the same order: the FP32 oracle bit for bit
            assert np.array_equal(x32, _oracle_f32(orc, lv, ip, pf, c_ai, c_aj, c_av, d, b))
            monkeypatch.setenv("LA_TRSV_SCHEDULE", "flags" if schedule == "parts" else "parts")
            _, y32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
            monkeypatch.setenv("LA_TRSV_SCHEDULE", schedule)
            assert np.array_equal(x32, y32), (n, uplo, "fp32 schedules differ")


def _oracle_f32(orc, lv, ip, pf, c_ai, c_aj, c_av, d, b):
    """The oracle's FP32 level solve (float storage, one float operation per
    step, the reference's row order), as float64 for comparison."""
    P = orc.ptr
    n = len(c_ai) - 1
    b32 = np.ascontiguousarray(b, np.float32)
    x = np.zeros(n, np.float32)
    orc.port().oracle_level_solve_f32(lv, P(ip), P(pf), 0, P(c_ai), P(c_aj), P(c_av),
                                      P(None if d is None else np.ascontiguousarray(d)),
                                      P(b32), P(x))
    return x.astype(np.float64)


def test_trsv_second_row_variant_bit_identical(lab, orc, monkeypatch):
    """The partitioned FP32 kernel with second-row register sets (W2), which
    the analysis picks for 3-slot FP32 factors when some level of a part is
    wider than the CTA -- the variant the large anisotropic PCG's FP32 solves
    run.  Two parts on RCM-ordered 40^3 / 48^3 IC(0) factors make the parts'
    levels wider than 512 rows, so W2 is provably selected; its solve equals
    the FP32 oracle bit for bit, the partitioned kernel without W2
    (LA_TRSV_W2=0) bit for bit, and the FP64 oracle within 1e-4."""
    from linearalgebra_b200 import gen
    P = orc.ptr
    monkeypatch.setenv("LA_TRSV_SCHEDULE", "parts")
    monkeypatch.setenv("LA_TRSV_PARTS", "2")
    monkeypatch.delenv("LA_TRSV_W2", raising=False)
    checked = 0
    for n, ai, aj, av in (gen.laplacian_3d(40), gen.aniso7(48, seed=2)):
        _, lt, ut, d = _ic_factor_rcm(lab, n, ai, aj, av)
        for uplo, (c_ai, c_aj, c_av) in (("L", lt), ("U", ut)):
            b = np.random.default_rng(n + 11).uniform(-1, 1, n)
            ts32, x32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
            assert ts32.schedule() == ("parts", 2), ts32.schedule()
            assert ts32.variant() == (3, True), ts32.variant()
            lv, ip, pf = ts32.levels()
            assert np.array_equal(x32, _oracle_f32(orc, lv, ip, pf, c_ai, c_aj, c_av, d, b)), \
                (n, uplo)
            ref = np.zeros(n)
            orc.port().oracle_level_solve(lv, P(ip), P(pf), 0, P(c_ai), P(c_aj), P(c_av),
                                          P(d), P(b), P(ref))
            e = rel(x32, ref)
            print(f"W2 n={n} {uplo}: fp32 err vs fp64 oracle {e:.2e}")
            assert e <= 1e-4
            monkeypatch.setenv("LA_TRSV_W2", "0")
            ts1, y32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
            monkeypatch.delenv("LA_TRSV_W2")
            assert ts1.variant() == (3, False)
            assert np.array_equal(x32, y32), (n, uplo, "W2 differs from one register set")
            checked += 1
    assert checked == 4


def test_reference_free_solves_bit_exact(lab, orc, golden):
    """The reference's free functions with their host-array signatures --
    ForwardSubstitution, BackwardSubstitution and the two level-scheduled
    forms (triangle_solve.hpp:32-145) -- each planned and solved on the GPU:
    bit for bit the compiled reference's results (the oracle's where the
    reference library is absent)."""
    P = orc.ptr
    rf = orc.ref()
    port = orc.port()
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if m != n:
            continue
        l_ai, l_aj, l_av = strict_triangle(n, ai, aj, av, True)
        u_ai, u_aj, u_av = strict_triangle(n, ai, aj, av, False)
        rng = np.random.default_rng(n + 3)
        b = rng.uniform(-1, 1, n)
        d = rng.uniform(1, 2, n)
        want = np.zeros(n)
        (rf.la_ref_forward_substitution if rf else port.oracle_forward_substitution)(
            n, 0, P(l_ai), P(l_aj), P(l_av), P(b), P(want))
        got = lab.ForwardSubstitution(n, 0, l_ai, l_aj, l_av, b, np.zeros(n))
        assert np.array_equal(got, want, equal_nan=True), (name, "forward")
        want = np.zeros(n)
        (rf.la_ref_backward_substitution if rf else port.oracle_backward_substitution)(
            n, 0, P(u_ai), P(u_aj), P(u_av), P(d), P(b), P(want))
        got = lab.BackwardSubstitution(n, 0, u_ai, u_aj, u_av, d, b, np.zeros(n))
        assert np.array_equal(got, want, equal_nan=True), (name, "backward")
        if rf:
            lv, ip, pf = lab.TopologicalSort2("L", n, 0, l_ai, l_aj)
            want = np.zeros(n)
            rf.la_ref_level_forward(4, P(ip), P(pf), lv, n, 0, P(l_ai), P(l_aj), P(l_av),
                                    P(b), P(want))
            got = lab.LevelScheduleForwardSubstitution(ip, pf, lv, n, 0, l_ai, l_aj, l_av, b,
                                                       np.zeros(n))
            assert np.array_equal(got, want, equal_nan=True), (name, "level forward")
            lv, ip, pf = lab.TopologicalSort2("U", n, 0, u_ai, u_aj)
            want = np.zeros(n)
            rf.la_ref_level_backward(4, P(ip), P(pf), lv, n, 0, P(u_ai), P(u_aj), P(u_av),
                                     P(d), P(b), P(want))
            got = lab.LevelScheduleBackwardSubstitution(ip, pf, lv, n, 0, u_ai, u_aj, u_av,
                                                        d, b, np.zeros(n))
            assert np.array_equal(got, want, equal_nan=True), (name, "level backward")
        checked += 1
    assert checked >= 5


def test_ilu0_apply_bit_exact(lab, orc):
    """The ILU apply (incomplete_lu.cpp:36-48): la_ilu0's factor split by
    SplitLDU, a unit-lower then an upper solve on the GPU -- bit for bit the
    oracle's ForwardSubstitution / BackwardSubstitution of the same factor,
    on 3D stencils and a nonsymmetric random pattern."""
    from linearalgebra_b200 import gen
    P = orc.ptr
    rng = np.random.default_rng(21)
    mats = [gen.laplacian_3d(16), gen.aniso7(12, seed=5)]
    m = 2000  # nonsymmetric, diagonally dominant
    rows = [np.union1d(rng.choice(m, 6, replace=False), [i]) for i in range(m)]
    ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    aj = np.concatenate(rows).astype(np.int32)
    av = rng.uniform(-1, 1, len(aj))
    r = np.repeat(np.arange(m), np.diff(ai))
    av[aj == r] = 8.0
    mats.append((m, ai, aj, av))
    for n, ai, aj, av in mats:
        lu = lab.ILU0(n, 0, ai, aj, av)
        (l_ai, l_aj, l_av), d, (u_ai, u_aj, u_av) = lab.SplitLDU(n, 0, ai, aj, lu)
        b = rng.uniform(-1, 1, n)
        t = lab.ForwardSubstitution(n, 0, l_ai, l_aj, l_av, b, np.zeros(n))
        x = lab.BackwardSubstitution(n, 0, u_ai, u_aj, u_av, d, t, np.zeros(n))
        t_ref = np.zeros(n)
        orc.port().oracle_forward_substitution(n, 0, P(l_ai), P(l_aj), P(l_av), P(b), P(t_ref))
        x_ref = np.zeros(n)
        orc.port().oracle_backward_substitution(n, 0, P(u_ai), P(u_aj), P(u_av), P(d), P(t_ref),
                                                P(x_ref))
        assert np.array_equal(t, t_ref) and np.array_equal(x, x_ref), n


def test_forward_substitution_t(lab, orc, golden):
    """ForwardSubstitutionT (triangle_solve.hpp:87-98): the unit lower solve
    with L = U^T given as the CSR of the strict upper triangle U.  The GPU
    plans the transposed triangle; FP64 agrees with the oracle and with the
    compiled reference to <= 1e-13 (the reference subtracts each product in
    turn, the plan sums a row first), FP32 to 1e-4 where the solution stays
    within 1e3 of zero; with a diagonal it solves
    (U^T + D) x = b like the plain lower solve on an explicit transpose."""
    P = orc.ptr
    rf = orc.ref()
    from linearalgebra_b200 import gen
    mats = [(name, n, ai, aj, av) for name, m, n, ai, aj, av in golden_matrices(golden) if m == n]
    n3, a3, j3, v3 = gen.laplacian_3d(24)
    mats.append(("lap3d_24", n3, a3, j3, v3))
    checked = 0
    for name, n, ai, aj, av in mats:
        u_ai, u_aj, u_av = strict_triangle(n, ai, aj, av, False)
        b = np.random.default_rng(n).uniform(-1, 1, n)
        ref = np.zeros(n)
        orc.port().oracle_forward_substitution_t(n, 0, P(u_ai), P(u_aj), P(u_av), P(b), P(ref))
        if rf is not None:
            ref2 = np.zeros(n)
            rf.la_ref_forward_substitution_t(n, 0, P(u_ai), P(u_aj), P(u_av), P(b), P(ref2))
            assert np.array_equal(ref, ref2), name  # the oracle restates the reference
        x = np.zeros(n)
        lab.ForwardSubstitutionT(n, 0, u_ai, u_aj, u_av, b, x)
        assert rel(x, ref) <= TOL, (name, rel(x, ref))
        ts = lab.OptimizedTriangularSolve("L", dtype=np.float32).analysis_transposed(
            n, 0, u_ai, u_aj, u_av)
        x32 = torch.empty(n, dtype=torch.float32, device="cuda")
        ts(dev(b, torch.float32), x32)
        if np.abs(ref).max() <= 1e3:  # unit triangles can grow far beyond FP32's range
            assert rel(x32.double().cpu().numpy(), ref) <= 1e-4, name
        d = np.random.default_rng(n + 7).uniform(1, 2, n)
        tsd, xd = solve(lab, "L", n, *lab.Transpose(n, n, 0, u_ai, u_aj, u_av), d, b)
        ts2 = lab.OptimizedTriangularSolve("L").analysis_transposed(n, 0, u_ai, u_aj, u_av, d)
        y = torch.empty(n, dtype=torch.float64, device="cuda")
        ts2(dev(b), y)
        assert np.array_equal(y.cpu().numpy(), xd), name
        checked += 1
    assert checked >= 5


def _chain_with_skips(n, seed):
    """Strict lower triangle: row i reads rows i-1, i-500 and i-1500 (when
    they exist) -- one row per level, and dependencies far older than the
    levels just before."""
    r = np.random.default_rng(seed)
    cols = [[j for j in (i - 1500, i - 500, i - 1) if j >= 0] for i in range(n)]
    ai = np.concatenate([[0], np.cumsum([len(c) for c in cols])]).astype(np.int32)
    aj = np.concatenate([np.array(c, np.int64) for c in cols]).astype(np.int32)
    return ai, aj, r.uniform(-0.3, 0.3, int(ai[-1]))


def test_trsv_ring_bit_identical(lab, orc, monkeypatch):
    """The partitioned schedule with each part's x slots as a shared-memory
    ring (the form taken when a part's rows do not fit in shared memory),
    forced onto small cases: bit-identical to the oracle in both triangles
    and both precisions.  Cases: IC(0) factors with the default parts; the
    40^3 factor on 2 parts, whose levels are wider than a CTA (rows beyond
    the first per thread read b directly); a chain with skips on 3 parts and
    a 32-row ring, whose dependencies 500 and 1500 rows back are older than
    the ring and are read from x."""
    from linearalgebra_b200 import gen
    P = orc.ptr
    monkeypatch.setenv("LA_TRSV_SCHEDULE", "parts")
    cases = []
    for n, ai, aj, av in (gen.laplacian_3d(40), gen.aniso7(28, seed=3)):
        _, lt, ut, d = _ic_factor_rcm(lab, n, ai, aj, av)
        cases += [(n, "L", lt, d, None, ("1024", "2048", "4096")),
                  (n, "U", ut, d, None, ("1024", "2048", "4096"))]
        if n == 64_000:
            cases.append((n, "L", lt, d, "2", ("2048", "4096", "8192")))
    n = 3000
    cases.append((n, "L", _chain_with_skips(n, 4), np.random.default_rng(5).uniform(1, 2, n),
                  "3", ("32",)))
    for n, uplo, (c_ai, c_aj, c_av), d, parts, rings in cases:
        if parts:
            monkeypatch.setenv("LA_TRSV_PARTS", parts)
        else:
            monkeypatch.delenv("LA_TRSV_PARTS", raising=False)
        b = np.random.default_rng(n + 1).uniform(-1, 1, n)
        for ring in rings:  # the smallest ring that holds three levels
            monkeypatch.setenv("LA_TRSV_RING", ring)
            ts, x = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b)
            if ts.schedule()[0] == "parts-ring":
                break
        assert ts.schedule()[0] == "parts-ring", (n, uplo, parts, ts.schedule())
        lv, ip, pf = ts.levels()
        ref = np.zeros(n)
        orc.port().oracle_level_solve(lv, P(ip), P(pf), 0, P(c_ai), P(c_aj), P(c_av),
                                      P(d), P(b), P(ref))
        assert np.array_equal(x, ref), (n, uplo, parts, ring)
        ts32, x32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
        assert ts32.schedule()[0] == "parts-ring", (n, uplo, ts32.schedule())
        monkeypatch.delenv("LA_TRSV_RING")
        _, y32 = solve(lab, uplo, n, c_ai, c_aj, c_av, d, b, dtype=np.float32)
        assert np.array_equal(x32, y32), (n, uplo, "fp32 ring differs from whole parts")


def test_trsv_partitioned_is_chosen_for_3d_ic0(lab):
    """The analysis picks the partitioned schedule for the RCM-ordered IC(0)
    factor of the 128^3 Laplacian (the preconditioner of the PCG workload)."""
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_3d(128)
    _, (t_ai, t_aj, t_av), _, d = _ic_factor_rcm(lab, n, ai, aj, av)
    for dt in (np.float64, np.float32):
        ts = lab.OptimizedTriangularSolve("L", dtype=dt).analysis(n, 0, t_ai, t_aj, t_av, d)
        kind, parts = ts.schedule()
        assert kind == "parts" and parts > 1, (dt, kind, parts)
