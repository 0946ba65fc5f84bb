"""Matrix Market (coordinate) reader producing zero-based sorted CSR.

Stands in for the reference's reader (utils/utils.h:92-132, built on
fast_matrix_market): coordinate entries are sorted by (row, column) and
converted to CSR; `symmetric` / `skew-symmetric` / `hermitian` storage is
expanded to the full matrix (fast_matrix_market's default generalisation),
and `pattern` entries get the value 1.
"""
from __future__ import annotations

import numpy as np


def read_mtx(path):
    """Return (n_rows, n_cols, ai, aj, av) with int32 indices, float64 values."""
    with open(path, "r") as f:
        header = f.readline().split()
        if len(header) < 5 or header[0] != "%%MatrixMarket" or header[2] != "coordinate":
            raise ValueError(f"{path}: not a coordinate Matrix Market file")
        field, symm = header[3].lower(), header[4].lower()
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nz = (int(t) for t in line.split()[:3])
        data = np.loadtxt(f, ndmin=2) if nz else np.zeros((0, 3))
    r = data[:, 0].astype(np.int64) - 1
    c = data[:, 1].astype(np.int64) - 1
    v = np.ones(len(r)) if field == "pattern" else data[:, 2].astype(np.float64)
    if symm in ("symmetric", "skew-symmetric", "hermitian"):
        off = r != c
        sign = -1.0 if symm == "skew-symmetric" else 1.0
        r, c, v = (np.concatenate([r, c[off]]), np.concatenate([c, r[off]]),
                   np.concatenate([v, sign * v[off]]))
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    ai = np.zeros(m + 1, np.int64)
    np.add.at(ai, r + 1, 1)
    np.cumsum(ai, out=ai)
    return m, n, ai.astype(np.int32), c.astype(np.int32), v
