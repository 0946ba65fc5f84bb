"""Seeded synthetic matrices for the five benchmark configurations.

The reference benchmarks on downloaded SuiteSparse matrices (thermal2 and
others) that are not available here; these generators stand in for them
with the shapes, sizes and value distributions the configurations state.
All use numpy's PCG64 generator (``np.random.default_rng(seed)``); every
matrix is CSR, zero-based, int32 indices, rows sorted by column.

C1 laplacian_2d(512)            5-point, diag 4, off-diagonals -1
C2 powerlaw(4_000_000, seed=0)  row lengths ceil(Pareto(2.1) on [1, inf))
                                clipped to [1, 20000]; columns uniform
                                without replacement, sorted; values N(0,1)
C3 laplacian_3d(128)            7-point, diag 6, off-diagonals -1
C4 stencil27(96, seed=0)        off-diagonals -U[0.5,1.5] (symmetric),
                                diag = 1.05 * row abs-sum
C5 aniso7(192, seed=0)          face coefficients lognormal(0, 2), z faces
                                x100, Dirichlet faces on the boundary; SPD
"""
from __future__ import annotations

import numpy as np


def _csr_from_offsets(g_shape, offsets, vals_of=None, diag=None):
    """Assemble a stencil matrix on a grid of shape (nz, ny, nx) (or 2D).

    offsets: list of integer offset tuples, sorted so that column indices
    increase; values given per offset by vals_of(offset, mask) or a constant.
    """
    dims = len(g_shape)
    n = int(np.prod(g_shape))
    coords = np.indices(g_shape).reshape(dims, -1)
    strides = np.array([int(np.prod(g_shape[i + 1:])) for i in range(dims)])
    cols_list, vals_list, mask_list = [], [], []
    for off in offsets:
        nb = coords + np.array(off)[:, None]
        m = np.all((nb >= 0) & (nb < np.array(g_shape)[:, None]), axis=0)
        col = (np.arange(n) + int(np.dot(strides, off))).astype(np.int64)
        mask_list.append(m)
        cols_list.append(col)
        vals_list.append(vals_of(off, m))
    M = np.stack(mask_list, axis=1)           # n x k
    Ccols = np.stack(cols_list, axis=1)
    V = np.stack(vals_list, axis=1)
    counts = M.sum(axis=1)
    ai = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=ai[1:])
    aj = Ccols[M].astype(np.int32)
    av = V[M].astype(np.float64)
    return n, ai.astype(np.int32), aj, av


def laplacian_2d(g: int):
    offs = [(-1, 0), (0, -1), (0, 0), (0, 1), (1, 0)]
    def v(off, m):
        return np.full(m.shape, 4.0 if off == (0, 0) else -1.0)
    return _csr_from_offsets((g, g), offs, v)


def laplacian_3d(g: int):
    offs = [(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 0), (0, 0, 1),
            (0, 1, 0), (1, 0, 0)]
    def v(off, m):
        return np.full(m.shape, 6.0 if off == (0, 0, 0) else -1.0)
    return _csr_from_offsets((g, g, g), offs, v)


def stencil27(g: int, seed: int = 0):
    """SPD 27-point stencil: symmetric off-diagonals -U[0.5, 1.5] drawn per
    undirected edge, diagonal 1.05 x row abs-sum."""
    rng = np.random.default_rng(seed)
    n = g ** 3
    offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1)
            for dx in (-1, 0, 1)]
    # one value per (node, positive offset); negative offsets read the
    # value stored at the neighbour for the mirrored offset
    pos = [o for o in offs if o > (0, 0, 0)]
    edge = {o: -rng.uniform(0.5, 1.5, n) for o in pos}
    stride = np.array([g * g, g, 1])

    def v(off, m):
        if off == (0, 0, 0):
            return np.zeros(m.shape)
        if off > (0, 0, 0):
            return edge[off]
        mirror = tuple(-c for c in off)
        src = np.arange(n) + int(np.dot(stride, off))
        out = np.zeros(n)
        out[m] = edge[mirror][src[m]]
        return out

    n, ai, aj, av = _csr_from_offsets((g, g, g), offs, v)
    rows = np.repeat(np.arange(n), np.diff(ai))
    absum = np.bincount(rows, weights=np.abs(av), minlength=n)
    diag_pos = ai[:-1] + np.array([13] * n) - _missing_before_center(g, offs)
    av[diag_pos] = 1.05 * absum
    return n, ai, aj, av


def _missing_before_center(g, offs):
    """Per row, the number of out-of-grid offsets that precede the centre."""
    coords = np.indices((g, g, g)).reshape(3, -1)
    miss = np.zeros(coords.shape[1], np.int64)
    for off in offs:
        if off >= (0, 0, 0):
            break
        nb = coords + np.array(off)[:, None]
        ok = np.all((nb >= 0) & (nb < g), axis=0)
        miss += ~ok
    return miss


def aniso7(g: int, seed: int = 0, sigma: float = 2.0, zscale: float = 100.0):
    """Anisotropic 7-point finite-volume diffusion with lognormal face
    coefficients (z faces x zscale) and Dirichlet boundary faces: the
    diagonal is the sum of the node's six face coefficients (boundary faces
    included), so the matrix is SPD."""
    rng = np.random.default_rng(seed)
    n = g ** 3
    # face coefficients: fx[z, y, x] between x and x+1 for x in [-1, g-1]
    fx = rng.lognormal(0.0, sigma, (g, g, g + 1))
    fy = rng.lognormal(0.0, sigma, (g, g + 1, g))
    fz = rng.lognormal(0.0, sigma, (g + 1, g, g)) * zscale
    coef = {
        (0, 0, -1): fx[:, :, :-1], (0, 0, 1): fx[:, :, 1:],
        (0, -1, 0): fy[:, :-1, :], (0, 1, 0): fy[:, 1:, :],
        (-1, 0, 0): fz[:-1, :, :], (1, 0, 0): fz[1:, :, :],
    }
    diag = sum(c for c in coef.values()).reshape(-1)
    offs = [(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 0), (0, 0, 1),
            (0, 1, 0), (1, 0, 0)]

    def v(off, m):
        if off == (0, 0, 0):
            return diag
        return -coef[off].reshape(-1)

    return _csr_from_offsets((g, g, g), offs, v)


def powerlaw(n: int, seed: int = 0, exponent: float = 2.1,
             max_len: int = 20000, ncols: int | None = None):
    """Irregular rows: length ceil(X), X ~ Pareto with pdf ~ x^-exponent on
    [1, inf), clipped to [1, max_len]; columns uniform without replacement
    and sorted; values N(0, 1)."""
    rng = np.random.default_rng(seed)
    ncols = n if ncols is None else ncols
    u = rng.random(n)
    lens = np.ceil(u ** (-1.0 / (exponent - 1.0)))
    lens = np.clip(lens, 1, max_len).astype(np.int64)
    ai = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=ai[1:])
    nnz = int(ai[-1])
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, ncols, nnz, dtype=np.int64)
    # resample duplicates inside a row until none remain
    while True:
        key = rows * ncols + cols
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(nnz, bool)
        dup[order[1:][ks[1:] == ks[:-1]]] = True
        nd = int(dup.sum())
        if nd == 0:
            break
        cols[dup] = rng.integers(0, ncols, nd, dtype=np.int64)
    order = np.lexsort((cols, rows))
    aj = cols[order].astype(np.int32)
    av = rng.standard_normal(nnz)
    return n, ai.astype(np.int32), aj, av


def uniform_vector(n: int, seed: int = 0):
    """x ~ U[-1, 1] from `seed`."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def upper_with_diag(n, ai, aj, av):
    """Upper triangle incl. diagonal (SplitTriangle<U>) in numpy."""
    rows = np.repeat(np.arange(n), np.diff(ai))
    keep = aj >= rows
    cnt = np.bincount(rows[keep], minlength=n)
    u_ai = np.zeros(n + 1, np.int32)
    np.cumsum(cnt, out=u_ai[1:])
    return u_ai, aj[keep].astype(np.int32), av[keep].astype(np.float64)
