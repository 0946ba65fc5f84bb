"""RCM with large components ordered on the GPU (la_rcm_device): the same
(iperm, perm) as the host's la_rcm -- which equals the reference's SerialCM
(reordering/Reordering.cpp:37-136) on the golden fixtures -- on 2D / 3D
stencils above the device size threshold, with the nodes in natural and
shuffled numbering, and on a pattern of several components (a large one
between small ones and isolated nodes, ordered by their largest node)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relabel(n, ai, aj, av, seed):
    """The same graph with its nodes renumbered at random."""
    p = np.random.default_rng(seed).permutation(n).astype(np.int32)  # new -> old
    inv = np.argsort(p).astype(np.int32)
    import linearalgebra_b200 as la
    return la.Permute(n, 0, ai, aj, av, p, inv)


def _blocks(parts):
    """Block-diagonal union of (n, ai, aj, av) patterns."""
    ai_l, aj_l, off, nnz = [np.zeros(1, np.int64)], [], 0, 0
    for n, ai, aj, av in parts:
        ai_l.append(np.asarray(ai[1:], np.int64) + nnz)
        aj_l.append(np.asarray(aj, np.int64) + off)
        off += n
        nnz += int(ai[-1])
    return (off, np.concatenate(ai_l).astype(np.int32), np.concatenate(aj_l).astype(np.int32),
            np.ones(nnz))


def test_rcm_device_equals_host(lab):
    from linearalgebra_b200 import gen
    iso = (5, np.arange(6, dtype=np.int32), np.arange(5, dtype=np.int32), np.ones(5))
    cases = {
        "lap3d_48": gen.laplacian_3d(48),
        "st27_44": gen.stencil27(44, seed=1),
        "aniso_48": gen.aniso7(48, seed=4),
        "lap2d_400": gen.laplacian_2d(400),
        "multi": _blocks([gen.laplacian_2d(12), gen.laplacian_3d(44), iso, gen.laplacian_2d(3),
                          gen.laplacian_2d(300)]),
    }
    cases["lap3d_48_shuffled"] = (cases["lap3d_48"][0],
                                  *_relabel(*cases["lap3d_48"], seed=2))
    for name, (n, ai, aj, av) in cases.items():
        want = lab.SerialCM(n, 0, ai, aj)
        got = lab.SerialCM(n, 0, ai, aj, device=True)
        assert np.array_equal(got[0], want[0]), name
        assert np.array_equal(got[1], want[1]), name
        got1 = lab.SerialCM(n, 1, np.asarray(ai) + 1, np.asarray(aj) + 1, device=True)
        want1 = lab.SerialCM(n, 1, np.asarray(ai) + 1, np.asarray(aj) + 1)
        assert np.array_equal(got1[0], want1[0]), (name, "base 1")


def test_rcm_device_timing_c5_size(lab):
    """The 192^3 anisotropic diffusion pattern (C5): host and device
    orderings equal; prints both times."""
    import time
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.aniso7(192, seed=0)
    t0 = time.perf_counter()
    want = lab.SerialCM(n, 0, ai, aj)
    t_host = time.perf_counter() - t0
    lab.SerialCM(n, 0, ai, aj, device=True)
    t0 = time.perf_counter()
    got = lab.SerialCM(n, 0, ai, aj, device=True)
    t_dev = time.perf_counter() - t0
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    print(f"RCM 192^3: host {t_host:.3f} s, with the device ordering {t_dev:.3f} s")


def _random_connected(m, seed, max_extra=12):
    """A connected irregular symmetric pattern: a ring plus random chords
    (degrees 3 to ~40, many equal degrees, so the sweep's (degree, index)
    ties matter), diagonal included."""
    rng = np.random.default_rng(seed)
    i = np.arange(m)
    src = [i, (i + 1) % m]
    k = rng.integers(0, max_extra, m)
    a = np.repeat(i, k)
    b = rng.integers(0, m, len(a))
    keep = a != b
    rows = np.concatenate([i, i, (i + 1) % m, a[keep], b[keep]])
    cols = np.concatenate([i, (i + 1) % m, i, b[keep], a[keep]])
    key = np.unique(rows.astype(np.int64) * m + cols)
    r, c = key // m, (key % m).astype(np.int32)
    ai = np.zeros(m + 1, np.int32)
    np.cumsum(np.bincount(r, minlength=m), out=ai[1:])
    return m, ai, c


def test_rcm_device_irregular_graphs(lab):
    """Irregular connected graphs above the device threshold (every row at
    most 64 entries): the device ordering equals the host's, base 0 and 1."""
    for seed in range(3):
        n, ai, aj = _random_connected(70_000 + 5_000 * seed, seed)
        assert np.diff(ai).max() <= 64
        want = lab.SerialCM(n, 0, ai, aj)
        got = lab.SerialCM(n, 0, ai, aj, device=True)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), seed
        got1 = lab.SerialCM(n, 1, ai + 1, aj + 1, device=True)
        want1 = lab.SerialCM(n, 1, ai + 1, aj + 1)
        assert np.array_equal(got1[0], want1[0]) and np.array_equal(got1[1], want1[1]), seed


def test_rcm_device_rejects_what_the_host_rejects(lab):
    """The pattern check runs on the device for la_rcm_device: an
    unsymmetric pattern and a symmetric one with an unsorted row are both
    rejected, as la_rcm's transpose comparison rejects them."""
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_3d(42)  # 74,088 nodes: above the device threshold
    unsym_aj = aj.copy()
    r = 5000
    lo, hi = int(ai[r]), int(ai[r + 1])
    unsym_aj[hi - 1] = min(n - 1, int(unsym_aj[hi - 1]) + 1)  # (r, c) with no (c, r)
    unsorted_aj = aj.copy()
    unsorted_aj[lo], unsorted_aj[lo + 1] = aj[lo + 1], aj[lo]
    for bad in (unsym_aj, unsorted_aj):
        for dev in (False, True):
            with pytest.raises(lab.LAError) as e:
                lab.SerialCM(n, 0, ai, bad, device=dev)
            assert e.value.name == "LA_ERR_INVALID_ARG", dev
