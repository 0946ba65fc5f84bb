"""TopologicalSort2 on the GPU (la_topological_sort2_device): identical
outputs to the host's -- which equal the reference's TopologicalSort2
(matrix_utils.hpp:637-675) bit for bit -- for both triangles, base 0 and 1,
RCM-ordered and natural stencil factors, long rows and empty rows; entries
outside the strict triangle are rejected."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_matrices, strict_triangle

pytestmark = pytest.mark.gpu


def _random_lower(n, seed):
    r = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = 0 if i % 11 == 0 else (int(r.integers(20, 60)) if i % 501 == 7 else int(r.integers(0, 6)))
        k = min(k, i)
        rows.append(np.sort(r.choice(i, k, replace=False)) if k else np.zeros(0, np.int64))
    ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    return ai, (np.concatenate(rows) if ai[-1] else np.zeros(0)).astype(np.int32)


def test_levels_device_equal_host(lab, golden):
    from linearalgebra_b200 import gen
    cases = []
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if m == n:
            for lower in (True, False):
                t_ai, t_aj, _ = strict_triangle(n, ai, aj, av, lower)
                cases.append((name, "L" if lower else "U", n, t_ai, t_aj))
    for n, ai, aj, av in (gen.laplacian_3d(64), gen.stencil27(40), gen.aniso7(48, seed=2)):
        iperm, perm = lab.SerialCM(n, 0, ai, aj)
        b_ai, b_aj, b_av = lab.Permute(n, 0, ai, aj, av, iperm, perm)
        for lower in (True, False):
            t_ai, t_aj, _ = strict_triangle(n, b_ai, b_aj, b_av, lower)
            cases.append(("rcm", "L" if lower else "U", n, t_ai, t_aj))
        t_ai, t_aj, _ = strict_triangle(n, ai, aj, av, True)
        cases.append(("natural", "L", n, t_ai, t_aj))
    n = 200_000
    cases.append(("random", "L", n, *_random_lower(n, 3)))
    for name, uplo, n, t_ai, t_aj in cases:
        want = lab.TopologicalSort2(uplo, n, 0, t_ai, t_aj)
        got = lab.TopologicalSort2(uplo, n, 0, t_ai, t_aj, device=True)
        assert got[0] == want[0], (name, uplo)
        assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2]), (name, uplo)
        got1 = lab.TopologicalSort2(uplo, n, 1, t_ai + 1, t_aj + 1, device=True)
        want1 = lab.TopologicalSort2(uplo, n, 1, t_ai + 1, t_aj + 1)
        assert np.array_equal(got1[1], want1[1]) and np.array_equal(got1[2], want1[2])


def test_levels_device_rejects_non_strict(lab):
    ai = np.array([0, 1, 2], np.int32)
    aj = np.array([0, 0], np.int32)  # row 0 reads itself
    with pytest.raises(lab.LAError) as e:
        lab.TopologicalSort2("L", 2, 0, ai, aj, device=True)
    assert e.value.name == "LA_ERR_INVALID_ARG"


def test_partition_device_landmarks_equal_host(lab):
    """The partitioned solve's row partition with its landmark stage on the
    GPU (la_trsv_partition_device: the graph, the landmark searches and the
    candidate checks on the device, as the analysis computes it) equals the
    host's la_trsv_partition part for part -- grids in natural and RCM order,
    both triangles, a 27-point stencil, an anisotropic grid at full C3 size,
    a disconnected pattern (level coordinate only) and random triangles with
    base 1."""
    from linearalgebra_b200 import gen

    def strict(n, ai, aj, lower):
        r = np.repeat(np.arange(n), np.diff(ai))
        keep = (aj < r) if lower else (aj > r)
        t_ai = np.zeros(n + 1, np.int32)
        np.cumsum(np.bincount(r[keep], minlength=n), out=t_ai[1:])
        return t_ai, aj[keep].astype(np.int32)

    cases = []
    for name, (n, ai, aj, av), rcm in (("lap3d_20", gen.laplacian_3d(20), False),
                                       ("lap3d_24_rcm", gen.laplacian_3d(24), True),
                                       ("st27_12", gen.stencil27(12), False),
                                       ("aniso_16", gen.aniso7(16, seed=2), True),
                                       ("lap3d_128_rcm", gen.laplacian_3d(128), True)):
        if rcm:
            iperm, perm = lab.SerialCM(n, 0, ai, aj)
            ai, aj, av = lab.Permute(n, 0, ai, aj, av, iperm, perm)
        cases.append((name, n, np.asarray(ai, np.int32), np.asarray(aj, np.int32), 0))
    # two disjoint grids: not connected
    n1, a1, j1, _ = gen.laplacian_3d(10)
    ai = np.concatenate([a1, a1[1:] + a1[-1]]).astype(np.int32)
    aj = np.concatenate([j1, j1 + n1]).astype(np.int32)
    cases.append(("two_grids", 2 * n1, ai, aj, 0))
    rng = np.random.default_rng(3)
    m = 4000
    rows = [np.sort(rng.choice(m, 6, replace=False)) for _ in range(m)]
    r_ai = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    r_aj = np.concatenate(rows).astype(np.int32)
    cases.append(("random_base1", m, r_ai + 1, r_aj + 1, 1))
    for name, n, ai, aj, base in cases:
        for lower in (True, False):
            t_ai, t_aj = strict(n, ai - base, aj - base, lower)
            for nparts in (3, 148):
                uplo = "L" if lower else "U"
                want = lab.trsv_partition(uplo, n, base, t_ai + base, t_aj + base, nparts)
                got = lab.trsv_partition(uplo, n, base, t_ai + base, t_aj + base, nparts,
                                         device=True)
                assert got[1] == want[1] and np.array_equal(got[0], want[0]), \
                    (name, uplo, nparts, got[1], want[1])
