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
