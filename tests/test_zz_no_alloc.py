"""The allocation-free SpMV entry point (la_spmv_noalloc) against the
planned SpMV (la_spmv).

la_spmv_noalloc serves callers that must not allocate device memory --
code running under an application that hands out the whole device memory
budget through its own pool, or latency-critical loops that cannot take
cudaMalloc's implicit synchronisation -- by keeping its scratch in a fixed
device array.  Two calls in a row (different matrices, both reference forms)
must match the planned SpMV within the FP64 tolerance of the other SpMV tests
(1e-13 relative 2-norm); since both run the same kernels they are in fact
bit-identical.  The path it alone takes -- tile rows found on the device,
merge groups found by scanning them -- is also checked against the oracle
directly, and a CSR whose row pointers disagree with the declared nnz must
not make it write outside y.  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
TOL = 1e-13


def _dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dtype)


def _noalloc(lab, kind, n, ai_d, aj_d, av_d, nnz, alpha, x_d, beta, y_d):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lab._lib.call("la_spmv_noalloc", kind, n, nnz, 0, C.c_void_p(ai_d.data_ptr()),
                  C.c_void_p(aj_d.data_ptr()), C.c_void_p(av_d.data_ptr()), float(alpha),
                  C.c_void_p(x_d.data_ptr()), float(beta), C.c_void_p(y_d.data_ptr()), stream)


def test_noalloc_spmv_matches_planned_spmv_twice(lab, monkeypatch):
    """The allocation-free SpMV equals the planned tile pass bit for bit (the
    plan is held to the tile pass: the Laplacian would otherwise get the
    row-slot form, whose rows crossing a tile are summed in one piece)."""
    from linearalgebra_b200 import gen
    monkeypatch.setenv("LA_SPMV_ELL", "0")
    cases = [(lab.api.LA_SPMV_SEGSUM, gen.powerlaw(150_000, seed=4, max_len=4000), 1.0, 0.0),
             (lab.api.LA_SPMV_ALBUS, gen.laplacian_3d(48), -1.5, 0.5)]
    for kind, (n, ai, aj, av), alpha, beta in cases:
        nnz = int(ai[-1])
        rng = np.random.default_rng(n)
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, n)
        ai_d, aj_d = _dev(ai, torch.int32), _dev(aj, torch.int32)
        av_d, x_d = _dev(av, torch.float64), _dev(x, torch.float64)
        y_na = _dev(y0, torch.float64)
        _noalloc(lab, kind, n, ai_d, aj_d, av_d, nnz, alpha, x_d, beta, y_na)
        A = lab.CSR(n, n, 0, ai, aj, av)
        y_pl = _dev(y0, torch.float64)
        lab.SPMV(A, kind)(x_d, y_pl, alpha, beta)
        torch.cuda.synchronize()
        a, b = y_na.cpu().numpy(), y_pl.cpu().numpy()
        assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)
        assert np.array_equal(a, b)


def test_noalloc_rejects_inputs_beyond_its_scratch(lab):
    big = 32768 * 1024 + 1  # LA_SPMV_NOALLOC_MAX_NNZ + 1
    ai_d = torch.zeros(3, dtype=torch.int32, device="cuda")
    x_d = torch.zeros(2, dtype=torch.float64, device="cuda")
    y_d = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pytest.raises(lab.LAError) as e:
        _noalloc(lab, lab.api.LA_SPMV_SEGSUM, 2, ai_d, ai_d, x_d, big, 1.0, x_d, 0.0, y_d)
    assert e.value.name == "LA_ERR_INVALID_ARG"


def _oracle_cases():
    """(name, n, ai, aj, av): edge shapes (empty rows, rows on tile edges,
    rows spanning many tiles) and stencils, all rows short except where
    noted."""
    from linearalgebra_b200 import gen
    rng = np.random.default_rng(8)
    out = []
    for name, lens in (("empty_rows_tile_edges",
                        [0, 0, 3, 0, 2048, 0, 0, 1, 2047, 2049, 0, 5000, 1, 0, 4096, 7, 0, 0]),
                       ("sparse_rows", [0] * 5000 + [1] + [0] * 7000 + [2] + [0] * 3)):
        n = len(lens)
        ncols = 25000
        ai = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        aj = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]
                            ).astype(np.int32)
        out.append((name, n, ncols, ai, aj, rng.standard_normal(int(ai[-1]))))
    for name, (n, ai, aj, av) in (("lap3d_40", gen.laplacian_3d(40)),
                                  ("powerlaw_short", gen.powerlaw(60_000, seed=9, max_len=60))):
        out.append((name, n, n, ai, aj, av))
    return out


def test_noalloc_spmv_vs_oracle(lab, orc):
    """Against the oracle itself: bit for bit the reference's SegSum / ALBUS
    algorithm run over the 1024-nonzero tiles when every in-tile row segment
    is at most 64 long (the rows summed one per thread), and within 1e-13 of
    SerialSPMV on every case (long rows are summed by a warp)."""
    P = orc.ptr
    rng = np.random.default_rng(3)
    for name, n, ncols, ai, aj, av in _oracle_cases():
        x = rng.uniform(-1, 1, ncols)
        y0 = rng.uniform(-1, 1, n)
        seg = np.diff(ai)
        short = bool(np.all(seg <= 64))
        for kind, kname in ((lab.api.LA_SPMV_SEGSUM, "segsum"), (lab.api.LA_SPMV_ALBUS, "albus")):
            for alpha, beta in ((1.0, 0.0), (-1.5, 0.5)):
                ai_d, aj_d = _dev(ai, torch.int32), _dev(aj, torch.int32)
                av_d, x_d, y_d = _dev(av, torch.float64), _dev(x, torch.float64), \
                    _dev(y0, torch.float64)
                _noalloc(lab, kind, n, ai_d, aj_d, av_d, int(ai[-1]), alpha, x_d, beta, y_d)
                torch.cuda.synchronize()
                y = y_d.cpu().numpy()
                ser = y0.copy()
                orc.port().oracle_serial_spmv(n, 0, P(ai), P(aj), P(av), P(x), P(ser), alpha,
                                              beta)
                assert np.linalg.norm(y - ser) <= TOL * np.linalg.norm(ser), (name, kname)
                if short:
                    ref = y0.copy()
                    getattr(orc.port(), f"oracle_{kname}_spmv_tiled")(
                        1024, n, 0, P(ai), P(aj), P(av), P(x), P(ref), alpha, beta)
                    # ALBUSSPMV leaves the rows before its first block's start
                    # row unwritten (spmv.hpp:239-293); the GPU writes beta*y
                    # there as SerialSPMV does, checked above
                    lead = int(np.argmax(seg > 0)) if kname == "albus" else 0
                    assert np.array_equal(y[lead:], ref[lead:]), (name, kname, alpha, beta)


def test_noalloc_inconsistent_row_pointers_stay_inside_y(lab):
    """The caller's row pointers are not validated on the host.  With a
    declared nnz above ai[n] - base, or ai[0] above base, the result is
    undefined but no write may leave y[0, n): y sits inside a larger buffer
    whose guard entries before and after it must keep their values.  (The
    aj / av buffers hold the declared nnz entries, so every read is in
    bounds.)"""
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_3d(24)
    nnz = int(ai[-1])
    x_d = _dev(np.random.default_rng(1).uniform(-1, 1, n), torch.float64)
    guard = 64
    for kind in (lab.api.LA_SPMV_SEGSUM, lab.api.LA_SPMV_ALBUS):
        for case in ("nnz_too_large", "ai0_above_base"):
            extra = 3000
            aj_pad = np.concatenate([aj, np.zeros(extra, np.int32)])
            av_pad = np.concatenate([av, np.ones(extra)])
            if case == "nnz_too_large":
                ai_c, decl = ai, nnz + extra
            else:
                ai_c, decl = ai + 5, nnz
            buf = torch.full((n + 2 * guard,), 12345.0, dtype=torch.float64, device="cuda")
            y_d = buf[guard:guard + n]
            _noalloc(lab, kind, n, _dev(ai_c, torch.int32), _dev(aj_pad, torch.int32),
                     _dev(av_pad, torch.float64), decl, 1.0, x_d, 0.0, y_d)
            torch.cuda.synchronize()
            b = buf.cpu().numpy()
            assert np.all(b[:guard] == 12345.0) and np.all(b[guard + n:] == 12345.0), \
                (kind, case)
