"""GPU SpMV parity: both reference forms through the C-ABI vs the oracle.

Tolerance (FP64): relative 2-norm error <= 1e-13 against the reference's
serial result, plus an element-wise bound.  FP32
results state their error against the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_matrices

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
TOL = 1e-13
KINDS = ("segsum", "albus")


def kind_id(lab, k):
    return lab.api.LA_SPMV_SEGSUM if k == "segsum" else lab.api.LA_SPMV_ALBUS


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dtype)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def run_spmv(lab, m, n, ai, aj, av, x, y0, alpha, beta, kind, base=0):
    A = lab.CSR(m, n, base, ai, aj, av)
    plan = lab.SPMV(A, kind_id(lab, kind))
    xd, yd = dev(x), dev(y0)
    plan(xd, yd, alpha, beta)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def oracle_serial(orc, m, ai, aj, av, x, y0, alpha, beta, base=0):
    y = np.array(y0, dtype=np.float64, copy=True)
    P = orc.ptr
    orc.port().oracle_serial_spmv(m, base, P(ai), P(aj), P(av), P(x), P(y), alpha, beta)
    return y


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_golden(lab, golden, kind):
    for name, m, n, ai, aj, av in golden_matrices(golden):
        x, y0 = golden[f"{name}/spmv_x"], golden[f"{name}/spmv_y0"]
        ref = golden[f"{name}/spmv_serial"]
        y = run_spmv(lab, m, n, ai, aj, av, x, y0, 1.5, 0.5, kind)
        assert rel(y, ref) <= TOL, (name, rel(y, ref))
        assert np.all(np.abs(y - ref) <= 1e-12 * (np.abs(ref) + np.abs(y0) + 1)), name
        # the reference's own test vector: b = ones, alpha 1, beta 0
        y = run_spmv(lab, m, n, ai, aj, av, np.ones(n), np.zeros(m), 1.0, 0.0, kind)
        assert rel(y, golden[f"{name}/spmv_ones"]) <= TOL, name
        # the multi-threaded reference forms agree with the GPU as well
        for T in (7, 10):
            assert rel(run_spmv(lab, m, n, ai, aj, av, x, y0, 1.5, 0.5, kind),
                       golden[f"{name}/spmv_{kind}_T{T}"]) <= TOL


TILE = 1024       # nonzeros per GPU tile (la_spmv.cu kTile)
LONG_SEG = 64     # in-tile row segments longer than this use a warp sum


def short_segments_only(ai):
    """True when every row's part inside every 1024-nonzero tile is <= 64
    long (then each GPU row sum runs in the reference's sequential order)."""
    ai = ai.astype(np.int64)
    for r in range(len(ai) - 1):
        lo, hi = ai[r], ai[r + 1]
        while lo < hi:
            end = min(hi, (lo // TILE + 1) * TILE)
            if end - lo > LONG_SEG:
                return False
            lo = end
    return True


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_bit_exact_vs_tiled_reference_algorithm(lab, orc, golden, kind):
    """With the reference's SegSum / ALBUS algorithm run over the GPU's
    1024-nonzero chunks, the GPU result is bit-identical; rows that do not
    cross a tile are bit-identical to SerialSPMV (ALBUS form)."""
    P = orc.ptr
    fn = getattr(orc.port(), f"oracle_{kind}_spmv_tiled")
    checked = 0
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if not short_segments_only(ai) or ai[1] == ai[0]:
            continue
        x, y0 = golden[f"{name}/spmv_x"], golden[f"{name}/spmv_y0"]
        for alpha, beta, xv, yv in ((1.5, 0.5, x, y0), (1.0, 0.0, np.ones(n), np.zeros(m))):
            ref = yv.copy()
            fn(TILE, m, 0, P(ai), P(aj), P(av), P(xv), P(ref), alpha, beta)
            y = run_spmv(lab, m, n, ai, aj, av, xv, yv, alpha, beta, kind)
            assert np.array_equal(y, ref), (name, kind, alpha, np.abs(y - ref).max())
            if kind == "albus":
                ser = oracle_serial(orc, m, ai, aj, av, xv, yv, alpha, beta)
                inside = (ai[:-1] // TILE == np.maximum(ai[1:] - 1, ai[:-1]) // TILE)
                assert np.array_equal(y[inside], ser[inside]), name
        checked += 1
    assert checked >= 6


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_host_path_drop_in(lab, golden, kind):
    cls = lab.SegSumSPMV if kind == "segsum" else lab.ALBUSSPMV
    for name, m, n, ai, aj, av in golden_matrices(golden):
        if m != n:
            continue
        s = cls(10)
        s.preprocess(m, 0, ai, aj, av)
        x = golden[f"{name}/spmv_x"]
        y = golden[f"{name}/spmv_y0"].copy()
        s(m, 0, ai, aj, av, x, y, 1.5, 0.5)
        assert rel(y, golden[f"{name}/spmv_serial"]) <= TOL, name


def _edge_matrices():
    rng = np.random.default_rng(42)
    out = []
    # leading, trailing and interior empty rows, rows ending on tile edges
    lens = [0, 0, 3, 0, 2048, 0, 0, 1, 2047, 2049, 0, 5000, 1, 0, 4096, 7, 0, 0]
    out.append(("empty_rows_tile_edges", lens))
    # one huge row spanning many tiles between tiny rows
    out.append(("long_row", [1, 2, 20000, 3, 1]))
    # a single row
    out.append(("single_row", [9000]))
    # many empty rows in one tile
    out.append(("sparse_rows", [0] * 5000 + [1] + [0] * 7000 + [2] + [0] * 3))
    mats = []
    for name, lens in out:
        m = len(lens)
        ncols = 25000
        ai = np.zeros(m + 1, np.int64)
        np.cumsum(lens, out=ai[1:])
        aj = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]
                            if sum(lens) else [np.zeros(0, np.int64)])
        av = rng.standard_normal(int(ai[-1]))
        mats.append((name, m, ncols, ai.astype(np.int32), aj.astype(np.int32), av))
    return mats


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_edge_cases(lab, orc, kind):
    rng = np.random.default_rng(1)
    for name, m, n, ai, aj, av in _edge_matrices():
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, m)
        for alpha, beta in ((1.0, 0.0), (-2.0, 0.75), (0.5, 1.0)):
            y = run_spmv(lab, m, n, ai, aj, av, x, y0, alpha, beta, kind)
            ref = oracle_serial(orc, m, ai, aj, av, x, y0, alpha, beta)
            assert rel(y, ref) <= TOL, (name, alpha, beta, rel(y, ref))
    # nnz == 0: y = beta * y
    ai = np.zeros(6, np.int32)
    y = run_spmv(lab, 5, 5, ai, np.zeros(0, np.int32), np.zeros(0), np.ones(5), np.arange(5.0),
                 2.0, 0.5, kind)
    assert np.array_equal(y, 0.5 * np.arange(5.0))


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_host_path_chunks_bit_identical(lab, kind):
    """The host-pointer call runs the plan's tiles in up to 8 chunks and copies
    each chunk's finished rows out while the next runs: bit for bit the
    device call's result, including rows that span chunk edges (power-law
    rows up to 20,000 long; one 20,000-long row among tiny ones), empty rows
    on tile edges, and beta != 0 with y in place."""
    from linearalgebra_b200 import gen
    rng = np.random.default_rng(5)
    n, ai, aj, av = gen.powerlaw(200_000, seed=3)
    mats = [("powerlaw_200k", n, n, ai, aj, av)] + _edge_matrices()
    for name, m, n, ai, aj, av in mats:
        A = lab.CSR(m, n, 0, ai, aj, av)
        plan = lab.SPMV(A, kind_id(lab, kind))
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, m)
        for alpha, beta in ((1.0, 0.0), (-1.5, 0.5)):
            yd = dev(y0)
            plan(dev(x), yd, alpha, beta)
            yh = y0.copy()
            plan(x, yh, alpha, beta)
            assert np.array_equal(yh, yd.cpu().numpy()), (name, kind, alpha, beta)


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_beta_zero_does_not_read_y_and_base1(lab, orc, golden, kind):
    ai, aj, av = golden["rdist1/ai"], golden["rdist1/aj"], golden["rdist1/av"]
    n = len(ai) - 1
    x = golden["rdist1/spmv_x"]
    y0 = np.full(n, np.nan)
    y = run_spmv(lab, n, n, ai, aj, av, x, y0, 1.0, 0.0, kind)
    assert np.all(np.isfinite(y))
    ref = oracle_serial(orc, n, ai, aj, av, x, np.zeros(n), 1.0, 0.0)
    assert rel(y, ref) <= TOL
    # one-based indices give the same result
    y1 = run_spmv(lab, n, n, ai + 1, aj + 1, av, x, np.zeros(n), 1.0, 0.0, kind, base=1)
    assert rel(y1, ref) <= TOL


@pytest.mark.parametrize("kind", KINDS)
def test_spmv_deterministic(lab, golden, kind):
    ai, aj, av = golden["powerlaw_3000/ai"], golden["powerlaw_3000/aj"], golden["powerlaw_3000/av"]
    n = len(ai) - 1
    A = lab.CSR(n, n, 0, ai, aj, av)
    plan = lab.SPMV(A, kind_id(lab, kind))
    xd = dev(golden["powerlaw_3000/spmv_x"])
    outs = []
    for _ in range(5):
        yd = dev(golden["powerlaw_3000/spmv_y0"])
        plan(xd, yd, 1.5, 0.5)
        outs.append(yd.cpu().numpy())
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def test_spmv_full_size_configs(lab, orc):
    """C1 (2D Laplacian 512^2), C3 (3D Laplacian 128^3) and C2 (power law,
    4M rows) at full size, FP64 both forms vs the oracle; FP32 error stated."""
    from linearalgebra_b200 import gen
    for label, (n, ai, aj, av) in (("C1", gen.laplacian_2d(512)), ("C3", gen.laplacian_3d(128)),
                                   ("C2", gen.powerlaw(4_000_000, seed=0))):
        x = gen.uniform_vector(n, 0)
        ref = oracle_serial(orc, n, ai, aj, av, x, np.zeros(n), 1.0, 0.0)
        A = lab.CSR(n, n, 0, ai, aj, av, keep_f32=True)
        for kind in KINDS:
            plan = lab.SPMV(A, kind_id(lab, kind))
            yd = torch.empty(n, dtype=torch.float64, device="cuda")
            plan(dev(x), yd, 1.0, 0.0)
            e = rel(yd.cpu().numpy(), ref)
            assert e <= TOL, (label, kind, e)
            y32 = torch.empty(n, dtype=torch.float32, device="cuda")
            plan(dev(x, torch.float32), y32, 1.0, 0.0)
            e32 = rel(y32.double().cpu().numpy(), ref)
            print(f"{label} {kind}: fp64 rel err {e:.2e}; fp32 (values+vectors) rel err {e32:.2e}")
            assert e32 <= 1e-5, (label, kind, e32)


def test_spmv_adjoints(lab, orc, golden):
    """dL/dx = A^T g and dL/dvalues = g_i x_j, against the oracle."""
    P = orc.ptr
    for name, m, n, ai, aj, av in golden_matrices(golden):
        rng = np.random.default_rng(3)
        g = rng.standard_normal(m)
        x = rng.standard_normal(n)
        out0 = rng.standard_normal(n)
        A = lab.CSR(m, n, 0, ai, aj, av)
        plan = lab.SPMV(A)
        od = dev(out0)
        plan.transpose(dev(g), od, 0.75, 0.5)
        ref = out0.copy()
        orc.port().oracle_spmv_transpose(m, n, 0, P(ai), P(aj), P(av), P(g), P(ref), 0.75, 0.5)
        assert rel(od.cpu().numpy(), ref) <= TOL, name
        dv = torch.empty(len(aj), dtype=torch.float64, device="cuda")
        plan.sddmm(dev(g), dev(x), dv, -1.25)
        ref = np.empty(len(aj))
        orc.port().oracle_sddmm_pattern(m, 0, P(ai), P(aj), P(g), P(x), P(ref), -1.25)
        assert np.array_equal(dv.cpu().numpy(), ref), name


def test_sddmm_rows_found_in_every_tile_shape(lab, orc):
    """The sampled outer product finds each nonzero's row by a scan of the
    tile's row starts, or -- for tiles spanning more rows than shared memory
    holds (long runs of empty rows) -- by binary search: bit for bit the
    oracle on edge shapes (empty rows, rows on tile edges, rows spanning many
    tiles), a power-law matrix and a 27-point stencil."""
    from linearalgebra_b200 import gen
    P = orc.ptr
    mats = [(name, m, n, ai, aj, av) for name, m, n, ai, aj, av in _edge_matrices()]
    for name, t in (("powerlaw", gen.powerlaw(50_000, seed=6)), ("st27", gen.stencil27(20))):
        n, ai, aj, av = t
        mats.append((name, n, n, ai, aj, av))
    rng = np.random.default_rng(9)
    for name, m, n, ai, aj, av in mats:
        g, x = rng.standard_normal(m), rng.standard_normal(n)
        plan = lab.SPMV(lab.CSR(m, n, 0, ai, aj, av))
        dv = torch.empty(len(aj), dtype=torch.float64, device="cuda")
        plan.sddmm(dev(g), dev(x), dv, 0.5)
        ref = np.empty(len(aj))
        orc.port().oracle_sddmm_pattern(m, 0, P(ai), P(aj), P(g), P(x), P(ref), 0.5)
        assert np.array_equal(dv.cpu().numpy(), ref), name


def test_spmv_row_slot_form_bit_exact(lab, orc, monkeypatch):
    """The row-slot form the plan picks for large matrices of short rows:
    every row summed by one thread in stored order, so the result is the
    reference's algorithm over a single chunk (no row split) bit for bit --
    SegSum and ALBUS, several (alpha, beta), base 0 and 1, empty rows -- and
    the tile pass is used otherwise."""
    from linearalgebra_b200 import gen
    P = orc.ptr
    n0, ai0, aj0, av0 = gen.laplacian_3d(24)
    # a pattern with empty rows and rows of 1 to 8 entries, 80,000 rows
    rng = np.random.default_rng(9)
    m = 80_000
    lens = rng.integers(0, 9, m)
    lens[rng.choice(m, 500, replace=False)] = 0
    e_aj = np.concatenate([np.sort(rng.choice(m, k, replace=False)) for k in lens]).astype(np.int32)
    e_ai = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    e_av = rng.standard_normal(len(e_aj))
    # the ragged pattern pads by ~100% (mean row 4, longest 8): the plan keeps
    # the tile pass for it unless LA_SPMV_ELL=1 forces the row-slot form
    cases = [("lap3d_48", False, *gen.laplacian_3d(48)),
             ("aniso_44", False, *gen.aniso7(44, seed=2)),
             ("ragged_80k", True, m, e_ai, e_aj, e_av)]
    for name, force, n, ai, aj, av in cases:
        ai, aj = np.asarray(ai, np.int32), np.asarray(aj, np.int32)
        nnz = int(ai[-1])
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, n)
        if force:
            monkeypatch.delenv("LA_SPMV_ELL", raising=False)
            assert lab.SPMV(lab.CSR(n, n, 0, ai, aj, av)).layout() == 0, name
            monkeypatch.setenv("LA_SPMV_ELL", "1")
        for base in (0, 1):
            A = lab.CSR(n, n, base, ai + base, aj + base, av, keep_f32=True)
            for kind, kname in ((lab.api.LA_SPMV_SEGSUM, "segsum"),
                                (lab.api.LA_SPMV_ALBUS, "albus")):
                plan = lab.SPMV(A, kind)
                assert plan.layout() == int(np.diff(ai).max()), (name, plan.layout())
                for alpha, beta in ((1.0, 0.0), (1.5, 0.5), (-0.75, 2.0)):
                    y = torch_dev(y0)
                    plan(torch_dev(x), y, alpha, beta)
                    ref = y0.copy()
                    getattr(orc.port(), f"oracle_{kname}_spmv_tiled")(
                        max(nnz, 1), n, 0, P(ai), P(aj), P(av), P(x), P(ref), alpha, beta)
                    got = y.cpu().numpy()
                    # rows before the first stored entry: beta * y (the
                    # reference's chunked algorithms skip them, a quirk)
                    lead = int(np.argmax(np.diff(ai) > 0))
                    want_lead = np.zeros(lead) if beta == 0 else 0.0 + beta * y0[:lead]
                    assert np.array_equal(got[:lead], want_lead), (name, base, kname)
                    assert np.array_equal(got[lead:], ref[lead:]), (name, base, kname, alpha)
    # small matrices keep the tile pass
    monkeypatch.delenv("LA_SPMV_ELL", raising=False)
    A = lab.CSR(n0, n0, 0, ai0, aj0, av0)
    assert lab.SPMV(A).layout() == 0
    monkeypatch.setenv("LA_SPMV_ELL", "0")
    n, ai, aj, av = gen.laplacian_3d(48)
    assert lab.SPMV(lab.CSR(n, n, 0, ai, aj, av)).layout() == 0


def torch_dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda")


def test_spmv_xparts_emulated_ranks(lab):
    """The row-block SpMV of a sharded matrix reading x from its owners'
    slices (la_spmv_xparts), with the ranks emulated as separate device
    buffers on one GPU: bit-identical to the same block multiplied with the
    gathered x (la_spmv), for both forms and both precisions."""
    from linearalgebra_b200 import dist, gen
    for n, ai, aj, av in (gen.powerlaw(200_000, seed=4), gen.laplacian_3d(32)):
        x = gen.uniform_vector(n, 2)
        for world in (1, 3, 8):
            start = dist.row_blocks_by_nnz(ai, world)
            for dt in (torch.float64, torch.float32):
                xd = torch.as_tensor(x).to("cuda", dt)
                slices = [xd[int(start[r]):int(start[r + 1])].clone() for r in range(world)]
                for r in range(world):
                    r0, r1 = int(start[r]), int(start[r + 1])
                    bai, baj, bav = dist.block_rows(ai, aj, av, r0, r1)
                    A = lab.CSR(r1 - r0, n, 0, bai, baj, bav, keep_f32=True)
                    for kind in (lab.api.LA_SPMV_SEGSUM, lab.api.LA_SPMV_ALBUS):
                        plan = lab.SPMV(A, kind)
                        y1 = torch.full((r1 - r0,), 0.5, dtype=dt, device="cuda")
                        y2 = y1.clone()
                        plan(xd, y1, 1.25, 0.5)
                        plan.xparts(slices, start, y2, 1.25, 0.5)
                        assert torch.equal(y1, y2), (n, world, r, dt, kind)
    # argument checks
    n, ai, aj, av = gen.laplacian_2d(16)
    plan = lab.SPMV(lab.CSR(n, n, 0, ai, aj, av))
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(lab.LAError):
        plan.xparts([xd], [0, n - 1], y)          # must end at the column count
    with pytest.raises(lab.LAError):
        plan.xparts([xd] * 9, [0] * 9 + [n], y)  # more slices than allowed
