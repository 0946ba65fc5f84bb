"""Edge cases of the device preprocessing entry points: empty patterns,
one row, patterns without a single off-diagonal entry above the device
thresholds (no updates, no dependencies: one level), and isolated nodes
around a large component.  Every result equals the host's."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _diag_only(n):
    ai = np.arange(n + 1, dtype=np.int32)
    aj = np.arange(n, dtype=np.int32)
    return n, ai, aj, np.full(n, 4.0)


def test_factor_plan_empty_single_and_diagonal(lab):
    # n = 0: a plan and a numeric pass that do nothing
    ai0 = np.zeros(1, np.int32)
    aj0 = np.zeros(0, np.int32)
    for kind in ("ic0", "ilu0"):
        got = lab.FactorPlan(kind, 0, 0, ai0, aj0).factor(np.zeros(0))
        assert len(got) == 0
    # one row
    for kind, want in (("ic0", np.array([2.0])), ("ilu0", np.array([4.0]))):
        got = lab.FactorPlan(kind, 1, 0, np.array([0, 1], np.int32),
                             np.array([0], np.int32)).factor(np.array([4.0]))
        assert np.array_equal(got, want), kind
    # 70,000 diagonal rows: the device plan with no updates, one level
    n, ai, aj, av = _diag_only(70_000)
    want = lab.ICCLevelNumeric0(n, 0, ai, aj, av)
    plan = lab.FactorPlan("ic0", n, 0, ai, aj)
    assert plan.levels() == 1
    assert np.array_equal(plan.factor(av), want)
    assert np.array_equal(lab.FactorPlan("ilu0", n, 0, ai, aj).factor(av),
                          lab.ILU0(n, 0, ai, aj, av))


def test_levels_device_empty_and_without_dependencies(lab):
    for n in (0, 1, 70_000):
        ai = np.zeros(n + 1, np.int32)
        aj = np.zeros(0, np.int32)
        for uplo in ("L", "U"):
            want = lab.TopologicalSort2(uplo, n, 0, ai, aj)
            got = lab.TopologicalSort2(uplo, n, 0, ai, aj, device=True)
            assert got[0] == want[0] and np.array_equal(got[1], want[1])
            assert np.array_equal(got[2], want[2]), (n, uplo)


def test_rcm_device_empty_isolated_and_mixed(lab):
    from linearalgebra_b200 import gen
    # isolated nodes only (every component below the device threshold)
    for n in (0, 1, 70_000):
        ai = np.arange(n + 1, dtype=np.int32)
        aj = np.arange(n, dtype=np.int32)
        want = lab.SerialCM(n, 0, ai, aj)
        got = lab.SerialCM(n, 0, ai, aj, device=True)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), n
    # a large component with 5,000 isolated nodes before and after it
    n1, a1, j1, _ = gen.laplacian_3d(42)
    iso = 5000
    ai = np.concatenate([np.arange(iso + 1), a1[1:] + iso, a1[-1] + iso + np.arange(1, iso + 1)])
    aj = np.concatenate([np.arange(iso), j1 + iso, np.arange(iso + n1, 2 * iso + n1)])
    n = n1 + 2 * iso
    ai, aj = ai.astype(np.int32), aj.astype(np.int32)
    want = lab.SerialCM(n, 0, ai, aj)
    got = lab.SerialCM(n, 0, ai, aj, device=True)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_ingest_empty_and_single_entry(lab):
    for m, n in ((0, 0), (5, 7)):
        A = lab.csr_from_coo(m, n, 0, np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0))
        ai, aj, av = A.host
        assert np.array_equal(ai, np.zeros(m + 1, np.int32)) and len(aj) == 0 and len(av) == 0
    A = lab.csr_from_coo(3, 3, 1, np.array([3]), np.array([2]), np.array([1.5]))
    ai, aj, av = A.host
    assert list(ai) == [1, 1, 1, 2] and list(aj) == [2] and list(av) == [1.5]
