"""Ingest of the reference's on-disk formats (utils/utils.h:23-132).

CPU: the host readers through the C-ABI --
* la_read_binary_coo equals the reference's ReadFromBinaryCOO on its own
  data/shared/*.bin files (raw bytes frozen in tests/golden) entry for entry,
  including the (rows, cols) it returns, in both bases;
* la_read_matrix_market expands symmetric / skew-symmetric storage and
  pattern values as Matrix Market specifies, against a direct restatement;
* without a GPU the device builders fail loudly.
GPU: la_csr_read_binary_coo equals the reference's ReadFromBinaryCSR output
bit for bit, and the device sort (stable LSD radix by (row, col)) equals a
stable host sort on large shuffled inputs with duplicates, in both bases and
both value types; Matrix Market text reaches the same CSR.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available

REC = np.dtype([("v", "<f8"), ("c", "<i4"), ("r", "<i4")])  # std::tuple<int,int,double>


def write_bin(path, rows, cols, vals):
    rec = np.zeros(len(rows), REC)
    rec["r"], rec["c"], rec["v"] = rows, cols, vals
    with open(path, "wb") as f:
        f.write(np.int64(len(rows)).tobytes())
        f.write(rec.tobytes())


def golden_bins(golden, tmp_path):
    for nm in ("K", "M", "G", "G2"):
        p = tmp_path / f"{nm}.bin"
        p.write_bytes(golden[f"bin_{nm}/bytes"].tobytes())
        yield nm, p


def test_read_binary_coo_matches_reference_reader(lab, golden, tmp_path):
    """Entries in file order and the returned (rows, cols) = largest index
    + 1 - base, as ReadFromBinaryCOO (utils.h:23-44) returns them."""
    for nm, p in golden_bins(golden, tmp_path):
        raw = np.frombuffer(p.read_bytes(), REC, offset=8)
        for base in (1, 0):
            r, c, v, (m, n) = lab.ReadFromBinaryCOO(p, base)
            assert np.array_equal(r, raw["r"]) and np.array_equal(c, raw["c"])
            assert np.array_equal(v, raw["v"])
            assert (m, n) == tuple(golden[f"bin_{nm}/base{base}_shape"]), (nm, base)


def test_read_binary_coo_live_reference(lab, orc, tmp_path):
    """Against the compiled reference itself on a synthetic file (when the
    reference library was built here)."""
    rf = orc.ref()
    if rf is None:
        pytest.skip("compiled reference not available")
    rng = np.random.default_rng(3)
    rows, cols = rng.integers(1, 500, 3000), rng.integers(1, 700, 3000)
    p = tmp_path / "s.bin"
    write_bin(p, rows, cols, rng.standard_normal(3000))
    P = orc.ptr
    for base in (0, 1):
        m, n = np.zeros(1, np.int32), np.zeros(1, np.int32)
        cnt = rf.la_ref_read_binary_coo(str(p).encode(), base, None, None, None, P(m), P(n))
        rr, cc, vv = np.zeros(cnt, np.int32), np.zeros(cnt, np.int32), np.zeros(cnt)
        rf.la_ref_read_binary_coo(str(p).encode(), base, P(rr), P(cc), P(vv), P(m), P(n))
        r, c, v, mn = lab.ReadFromBinaryCOO(p, base)
        assert np.array_equal(r, rr) and np.array_equal(c, cc) and np.array_equal(v, vv)
        assert mn == (int(m[0]), int(n[0]))


def mm_text(m, n, rows, cols, vals, field="real", symm="general"):
    lines = [f"%%MatrixMarket matrix coordinate {field} {symm}", "% a comment",
             f"{m} {n} {len(rows)}"]
    for i, j, v in zip(rows, cols, vals):
        lines.append(f"{i + 1} {j + 1}" if field == "pattern" else f"{i + 1} {j + 1} {float(v)!r}")
    return "\n".join(lines) + "\n"


def expand(rows, cols, vals, symm):
    """Matrix Market's symmetric storage made general: every off-diagonal
    entry mirrored (negated for skew-symmetric), mirrors after the entry."""
    out = []
    for i, j, v in zip(rows, cols, vals):
        out.append((i, j, v))
        if symm != "general" and i != j:
            out.append((j, i, -v if symm == "skew-symmetric" else v))
    return [np.array([e[k] for e in out]) for k in range(3)]


@pytest.mark.parametrize("field,symm", [("real", "general"), ("real", "symmetric"),
                                        ("integer", "skew-symmetric"),
                                        ("pattern", "symmetric")])
def test_read_matrix_market_host(lab, tmp_path, field, symm):
    rng = np.random.default_rng(11)
    m = n = 400
    k = 2500
    rows, cols = rng.integers(0, m, k), rng.integers(0, n, k)
    if symm != "general":  # lower triangle, as symmetric files store it
        rows, cols = np.maximum(rows, cols), np.minimum(rows, cols)
        if symm == "skew-symmetric":
            keep = rows != cols
            rows, cols = rows[keep], cols[keep]
    vals = (rng.integers(-9, 9, len(rows)).astype(float) if field == "integer"
            else np.ones(len(rows)) if field == "pattern" else rng.standard_normal(len(rows)))
    p = tmp_path / "a.mtx"
    p.write_text(mm_text(m, n, rows, cols, vals, field, symm))
    mm, nn, r, c, v = lab.read_matrix_market_coo(p)
    er, ec, ev = expand(rows, cols, vals, symm)
    assert (mm, nn) == (m, n)
    assert np.array_equal(r, er) and np.array_equal(c, ec) and np.array_equal(v, ev)


def test_read_matrix_market_rejects_bad_input(lab, tmp_path):
    bad = {"banner.mtx": "%%NotMatrixMarket matrix coordinate real general\n1 1 1\n1 1 1\n",
           "array.mtx": "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
           "range.mtx": "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n"}
    for name, text in bad.items():
        p = tmp_path / name
        p.write_text(text)
        with pytest.raises(lab.LAError) as e:
            lab.read_matrix_market_coo(p)
        assert e.value.name == "LA_ERR_INVALID_ARG", name
    with pytest.raises(lab.LAError):
        lab.ReadFromBinaryCOO(tmp_path / "missing.bin")


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_device_ingest_fails_loudly_without_gpu(lab, golden, tmp_path):
    nm, p = next(golden_bins(golden, tmp_path))
    with pytest.raises(lab.LAError) as e:
        lab.ReadFromBinaryCSR(p, 1)
    assert e.value.name == "LA_ERR_NO_DEVICE"


# ------------------------------------------------------------------ GPU
def stable_csr(m, rows, cols, vals, base):
    """(ai, aj, av) of the entries stable-sorted by (row, col): the order the
    device sort gives (ties in input order)."""
    order = np.lexsort((cols, rows))  # lexsort is stable
    r = np.asarray(rows)[order] - base
    ai = np.zeros(m + 1, np.int64)
    np.add.at(ai, r + 1, 1)
    return ((np.cumsum(ai) + base).astype(np.int32), np.asarray(cols)[order].astype(np.int32),
            np.asarray(vals)[order])


@pytest.mark.gpu
def test_read_binary_csr_matches_reference(lab, golden, tmp_path):
    """ReadFromBinaryCSR (utils.h:46-91) on the reference's own files: the
    device CSR equals the reference's host CSR bit for bit, base 1 and 0."""
    for nm, p in golden_bins(golden, tmp_path):
        for base in (1, 0):
            A = lab.ReadFromBinaryCSR(p, base)
            key = f"bin_{nm}/base{base}"
            m, n = golden[f"{key}_shape"]
            assert (A.n, A.ncols, A.base) == (m, n, base), (nm, base)
            ai, aj, av = A.host
            assert np.array_equal(ai, golden[f"{key}_ai"]), (nm, base)
            assert np.array_equal(aj, golden[f"{key}_aj"]), (nm, base)
            assert np.array_equal(av, golden[f"{key}_av"]), (nm, base)


@pytest.mark.gpu
@pytest.mark.parametrize("base", [0, 1])
def test_device_coo_sort_large_shuffled(lab, base):
    """Shuffled entries with duplicates over index ranges that need several
    radix passes (and several scan levels): the device CSR equals a stable
    host sort; FP32 values follow the same order; an already ordered input
    (no sort) gives the same CSR; the CSR multiplies correctly."""
    import torch
    rng = np.random.default_rng(base)
    m, n, k = 70_000, 300_000, 1_500_000
    rows = rng.integers(0, m, k) + base
    cols = rng.integers(0, n, k) + base
    rows[-5000:], cols[-5000:] = rows[:5000], cols[:5000]  # duplicates, later in input
    vals = rng.standard_normal(k)
    A = lab.csr_from_coo(m, n, base, rows, cols, vals)
    want = stable_csr(m, rows, cols, vals, base)
    got = A.host
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    A32 = lab.csr_from_coo(m, n, base, rows, cols, vals.astype(np.float32), dtype=np.float32)
    assert np.array_equal(A32.host[2], want[2].astype(np.float32))
    B = lab.csr_from_coo(m, n, base, *[np.repeat(np.arange(m), np.diff(want[0])) + base,
                                       want[1], want[2]])
    for g, w in zip(B.host, want):
        assert np.array_equal(g, w)
    x = rng.uniform(-1, 1, n)
    y = torch.zeros(m, dtype=torch.float64, device="cuda")
    lab.SPMV(A)(torch.as_tensor(x).cuda(), y)
    r = np.repeat(np.arange(m), np.diff(want[0]))
    ref = np.bincount(r, weights=want[2] * x[want[1] - base], minlength=m)
    assert np.linalg.norm(y.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.gpu
def test_matrix_market_to_device_csr(lab, golden, tmp_path):
    """read_matrix_market_csr (utils.h:93-132): the golden matrices written
    as Matrix Market text (general, and their lower triangles as symmetric
    storage for the symmetric ones) come back as the same 0-based CSR."""
    from conftest import golden_matrices
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        rows = np.repeat(np.arange(m), np.diff(ai))
        p = tmp_path / f"{name}.mtx"
        p.write_text(mm_text(m, n, rows, aj, av))
        A = lab.read_matrix_market_csr(p)
        for g, w in zip(A.host, (ai, aj, av)):
            assert np.array_equal(g, w), name
        if m == n:
            dense_sym = True
            lower = aj <= rows
            mirror = dict(zip(zip(rows.tolist(), aj.tolist()), av.tolist()))
            dense_sym = all(mirror.get((c, r)) == v for r, c, v in
                            zip(rows.tolist(), aj.tolist(), av.tolist()))
            if dense_sym:
                p.write_text(mm_text(m, n, rows[lower], aj[lower], av[lower], "real", "symmetric"))
                B = lab.read_matrix_market_csr(p)
                for g, w in zip(B.host, (ai, aj, av)):
                    assert np.array_equal(g, w), (name, "symmetric")
        checked += 1
    assert checked >= 8
