"""IC(0) and ILU(0) numeric factorisation on the GPU (la_factor_*).

The device factor equals the host factorisation bit for bit -- la_icc0,
whose values are bit-identical to the reference's ICCLevelNumeric
(precond.hpp:615-693), and la_ilu0 -- on stencils in natural and RCM order,
a nonsymmetric pattern and base 1; a breakdown is reported at the row where
the sequential algorithm stops; the shift-retry loop (incomplete_cholesky.cpp
:315-342) ends at the same shift with the same factor.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available


def _ic_inputs(lab, mat, rcm):
    from linearalgebra_b200 import gen
    n, ai, aj, av = mat
    if rcm:
        iperm, perm = lab.SerialCM(n, 0, ai, aj)
        ai, aj, av = lab.Permute(n, 0, ai, aj, av, iperm, perm)
    ua, uj, uv = gen.upper_with_diag(n, ai, aj, av)
    return n, np.asarray(ua, np.int32), np.asarray(uj, np.int32), np.asarray(uv)


def _nonsym(m, seed, long_every=0):
    """Random nonsymmetric pattern, 6 off-diagonal entries a row (every
    long_every-th row 30: longer than the numeric pass's short-row form)."""
    rng = np.random.default_rng(seed)
    rows = [np.union1d(rng.choice(m, 30 if long_every and i % long_every == 0 else 6,
                                  replace=False), [i]) for i in range(m)]
    ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    aj = np.concatenate(rows).astype(np.int32)
    av = rng.uniform(-1, 1, len(aj))
    r = np.repeat(np.arange(m), np.diff(ai))
    av[aj == r] = 8.0
    return m, ai, aj, av


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_factor_plan_needs_a_device(lab):
    from linearalgebra_b200 import gen
    n, ua, uj, uv = _ic_inputs(lab, gen.laplacian_2d(8), False)
    with pytest.raises(lab.LAError) as e:
        lab.FactorPlan("ic0", n, 0, ua, uj)
    assert e.value.name == "LA_ERR_NO_DEVICE"


def test_ic0_plan_rejects_unsorted_rows(lab):
    """The IC(0) plan orders each row's updates from the pattern, which needs
    every row's columns strictly ascending from its diagonal: a row out of
    order, a repeated column or a column past n is rejected before any device
    work (so also without a GPU)."""
    from linearalgebra_b200 import gen
    n, ua, uj, uv = _ic_inputs(lab, gen.laplacian_2d(8), False)
    r = 5
    a, b = ua[r], ua[r + 1]
    assert b - a >= 3
    for bad in ("swap", "repeat", "past_n"):
        uj2 = uj.copy()
        if bad == "swap":
            uj2[a + 1], uj2[a + 2] = uj2[a + 2], uj2[a + 1]
        elif bad == "repeat":
            uj2[a + 2] = uj2[a + 1]
        else:
            uj2[b - 1] = n
        with pytest.raises(lab.LAError) as e:
            lab.FactorPlan("ic0", n, 0, ua, uj2)
        assert e.value.name == "LA_ERR_INVALID_ARG", bad


@pytest.mark.gpu
@pytest.mark.parametrize("rcm", [False, True])
def test_ic0_device_bit_identical(lab, rcm):
    from linearalgebra_b200 import gen
    for mat in (gen.laplacian_3d(32), gen.stencil27(16, seed=2), gen.aniso7(24, seed=1),
                gen.laplacian_2d(64)):
        n, ua, uj, uv = _ic_inputs(lab, mat, rcm)
        want = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
        plan = lab.FactorPlan("ic0", n, 0, ua, uj)
        got = plan.factor(uv)
        assert np.array_equal(got, want), (n, rcm, np.abs(got - want).max())
        # the same plan again, with a shift, and with device arrays
        import torch
        want2 = lab.ICCLevelNumeric0(n, 0, ua, uj, uv, omega=0.25)
        assert np.array_equal(plan.factor(uv, omega=0.25), want2)
        out = torch.empty(len(uv), dtype=torch.float64, device="cuda")
        plan.factor(torch.as_tensor(uv).cuda(), out=out)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want)


def _random_spd(m, seed):
    """An irregular symmetric M-matrix: random off-diagonal pattern (rows of
    1 to ~40 entries, a few long ones), negative off-diagonals, a dominant
    diagonal -- IC(0) exists, and the updates a row receives come in many
    different orders."""
    rng = np.random.default_rng(seed)
    rows = [set() for _ in range(m)]
    for i in range(m):
        k = rng.integers(0, 40) if rng.random() < 0.05 else rng.integers(0, 5)
        for j in rng.choice(m, k, replace=False):
            if j != i:
                rows[i].add(int(j))
                rows[j].add(i)
    ai = [0]
    aj, av = [], []
    for i in range(m):
        cols = sorted(rows[i] | {i})
        off = -rng.uniform(0.1, 1.0, len(cols))
        aj += cols
        av += list(off)
        ai.append(len(aj))
    ai, aj, av = np.array(ai, np.int32), np.array(aj, np.int32), np.array(av)
    r = np.repeat(np.arange(m), np.diff(ai))
    # symmetric values: the mean of (i, j) and (j, i), then a dominant diagonal
    key = np.minimum(r, aj).astype(np.int64) * m + np.maximum(r, aj)
    _, inv = np.unique(key, return_inverse=True)
    av = (np.bincount(inv, av) / np.bincount(inv))[inv]
    dsum = np.bincount(r, np.where(aj == r, 0.0, np.abs(av)), minlength=m)
    av[aj == r] = dsum + 1.0
    return m, ai, aj, av


@pytest.mark.gpu
def test_ic0_device_irregular_patterns(lab):
    """Irregular patterns, natural and RCM order: the device factor equals the
    host's bit for bit, so every row received its updates in the host's
    order."""
    for seed in range(4):
        for rcm in (False, True):
            n, ua, uj, uv = _ic_inputs(lab, _random_spd(4000 + 1000 * seed, seed), rcm)
            want = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
            got = lab.FactorPlan("ic0", n, 0, ua, uj).factor(uv)
            assert np.array_equal(got, want), (seed, rcm, np.abs(got - want).max())


def _arrow(m):
    """Tridiagonal plus a full last row and column, dominant diagonal: the
    last row receives m - 1 updates."""
    i = np.arange(m - 1)
    r = np.concatenate([i, i[1:], i[:-1], i, np.full(m - 1, m - 1), [m - 1]])
    c = np.concatenate([i, i[1:] - 1, i[:-1] + 1, np.full(m - 1, m - 1), i, [m - 1]])
    key = np.unique(r.astype(np.int64) * m + c)  # row-major, duplicates merged
    r, aj = (key // m).astype(np.int64), (key % m).astype(np.int32)
    ai = np.zeros(m + 1, np.int32)
    np.cumsum(np.bincount(r, minlength=m), out=ai[1:])
    av = np.where(aj == r, 0.0, -0.5)
    av[aj == r] = np.bincount(r, np.abs(av), minlength=m) + 1.0
    return m, ai, aj, av


@pytest.mark.gpu
def test_ic0_device_plan_large_patterns(lab):
    """From 65,536 rows the IC(0) plan itself is built on the device (update
    order, pairs, levels, chunks); the factor equals the host's bit for bit on
    stencils in natural and RCM order, an irregular pattern, base 1, and a
    pattern one of whose rows receives more updates than the device sorts
    (its plan is built on the host)."""
    from linearalgebra_b200 import gen
    cases = [("lap3d_48", gen.laplacian_3d(48), False), ("lap3d_48_rcm", gen.laplacian_3d(48), True),
             ("st27_42_rcm", gen.stencil27(42, seed=5), True),
             ("irregular_70k", _random_spd(70_000, 9), True), ("arrow_70k", _arrow(70_000), False)]
    for name, mat, rcm in cases:
        n, ua, uj, uv = _ic_inputs(lab, mat, rcm)
        assert n >= 65_536
        want = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
        plan = lab.FactorPlan("ic0", n, 0, ua, uj)
        got = plan.factor(uv)
        assert np.array_equal(got, want), (name, np.abs(got - want).max())
        if name == "lap3d_48_rcm":
            got1 = lab.FactorPlan("ic0", n, 1, ua + 1, uj + 1).factor(uv)
            assert np.array_equal(got1, want), name


@pytest.mark.gpu
@pytest.mark.parametrize("warp", ["0", "1"])
def test_factor_both_forms_bit_identical(lab, monkeypatch, warp):
    """The numeric pass in both forms -- a lane per row (LA_FACTOR_WARP=0)
    and a warp per row (=1; chosen by itself when rows receive more than 8
    pairs on average) -- on IC(0) of stencils (short and 27-point rows, in
    natural and RCM order), an irregular pattern with rows over 128 entries
    (their values worked on in global memory), ILU(0) with long rows, a
    shift, a breakdown and base 1: always the host's factor bit for bit."""
    from linearalgebra_b200 import gen
    monkeypatch.setenv("LA_FACTOR_WARP", warp)
    big = _random_spd(6000, 4)
    # one row of 200 entries: longer than the warp's shared slice
    n0, ai0, aj0, av0 = big
    rows = [list(aj0[ai0[i]:ai0[i + 1]]) for i in range(n0)]
    extra = np.random.default_rng(1).choice(np.arange(1, n0), 200, replace=False)
    for c in extra:
        if c not in rows[0]:
            rows[0].append(int(c))
            rows[int(c)].append(0)
    ai = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    aj = np.concatenate([sorted(r) for r in rows]).astype(np.int32)
    r = np.repeat(np.arange(n0), np.diff(ai))
    av = np.where(aj == r, 0.0, -0.3)
    av[aj == r] = np.bincount(r, np.abs(av), minlength=n0) + 1.0
    for name, mat, rcm in (("lap3d_24", gen.laplacian_3d(24), True),
                           ("st27_16", gen.stencil27(16, seed=2), False),
                           ("st27_16_rcm", gen.stencil27(16, seed=2), True),
                           ("long_rows", (n0, ai, aj, av), False)):
        n, ua, uj, uv = _ic_inputs(lab, mat, rcm)
        want = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
        plan = lab.FactorPlan("ic0", n, 0, ua, uj)
        assert np.array_equal(plan.factor(uv), want), (name, warp)
        want2 = lab.ICCLevelNumeric0(n, 0, ua, uj, uv, omega=0.25)
        assert np.array_equal(plan.factor(uv, omega=0.25), want2), (name, warp)
        got1 = lab.FactorPlan("ic0", n, 1, ua + 1, uj + 1).factor(uv)
        assert np.array_equal(got1, want), (name, warp, "base 1")
    # breakdown at the row where the sequential pass stops
    n, ua, uj, uv = _ic_inputs(lab, gen.stencil27(12, seed=3), False)
    j0 = n // 2
    bad = uv.copy()
    bad[ua[j0]] = 0.1
    with pytest.raises(lab.LAError):
        lab.ICCLevelNumeric0(n, 0, ua, uj, bad)
    with pytest.raises(lab.LAError) as e:
        lab.FactorPlan("ic0", n, 0, ua, uj).factor(bad)
    assert e.value.name == "LA_ERR_BREAKDOWN" and e.value.bad_row == j0, warp
    for n, ai, aj, av in (gen.laplacian_3d(16), _nonsym(2000, 6, long_every=5),
                          _nonsym(2000, 8, long_every=1)):
        want = lab.ILU0(n, 0, ai, aj, av)
        assert np.array_equal(lab.FactorPlan("ilu0", n, 0, ai, aj).factor(av), want), (n, warp)


@pytest.mark.gpu
def test_ic0_device_base1_and_breakdown(lab):
    from linearalgebra_b200 import gen
    n, ua, uj, uv = _ic_inputs(lab, gen.laplacian_3d(16), True)
    want = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    got = lab.FactorPlan("ic0", n, 1, ua + 1, uj + 1).factor(uv)
    assert np.array_equal(got, want)
    # a negative pivot at row j0 (its diagonal shrunk below what its updates
    # subtract): reported there; a shift large enough repairs it
    j0 = n // 3
    bad = uv.copy()
    bad[ua[j0]] = 0.1
    with pytest.raises(lab.LAError):
        lab.ICCLevelNumeric0(n, 0, ua, uj, bad)
    plan = lab.FactorPlan("ic0", n, 0, ua, uj)
    with pytest.raises(lab.LAError) as e:
        plan.factor(bad)
    assert e.value.name == "LA_ERR_BREAKDOWN" and e.value.bad_row == j0
    # shift retries: same shift, same factor as the host loop
    hv, hs = lab.ICCShifted(n, 0, ua, uj, bad)
    dv, ds = plan.shifted(bad)
    assert ds == hs and np.array_equal(dv, hv)


@pytest.mark.gpu
def test_ilu0_device_bit_identical(lab):
    from linearalgebra_b200 import gen
    for n, ai, aj, av in (gen.laplacian_3d(20), gen.aniso7(16, seed=3), _nonsym(3000, 5),
                          _nonsym(3000, 6, long_every=7)):
        want = lab.ILU0(n, 0, ai, aj, av)
        plan = lab.FactorPlan("ilu0", n, 0, ai, aj)
        assert np.array_equal(plan.factor(av), want), n
        got1 = lab.FactorPlan("ilu0", n, 1, np.asarray(ai) + 1, np.asarray(aj) + 1).factor(av)
        assert np.array_equal(got1, want), n
    # a zero pivot: row 1 of [[1, 1], [1, 1]]
    ai, aj = np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32)
    with pytest.raises(lab.LAError) as e:
        lab.FactorPlan("ilu0", 2, 0, ai, aj).factor(np.ones(4))
    assert e.value.bad_row == 1


@pytest.mark.gpu
def test_ic0_device_c3_size(lab):
    """The RCM-ordered 128^3 Laplacian's IC(0): bit-identical at full size;
    prints the host and device numeric times."""
    import time
    from linearalgebra_b200 import gen
    n, ua, uj, uv = _ic_inputs(lab, gen.laplacian_3d(128), True)
    t0 = time.perf_counter()
    want = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    t_host = time.perf_counter() - t0
    t0 = time.perf_counter()
    plan = lab.FactorPlan("ic0", n, 0, ua, uj)
    t_sym = time.perf_counter() - t0
    plan.factor(uv)
    t0 = time.perf_counter()
    got = plan.factor(uv)
    t_num = time.perf_counter() - t0
    assert np.array_equal(got, want)
    print(f"IC(0) 128^3: host {t_host * 1e3:.1f} ms, device plan {t_sym * 1e3:.1f} ms, "
          f"device numeric (host arrays in and out) {t_num * 1e3:.1f} ms, "
          f"{plan.levels()} levels")
