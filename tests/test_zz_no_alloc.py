"""The allocation-free SpMV entry point (la_spmv_noalloc) against the
planned SpMV (la_spmv).

la_spmv_noalloc serves callers that must not allocate device memory --
code running under an application that hands out the whole device memory
budget through its own pool, or latency-critical loops that cannot take
cudaMalloc's implicit synchronisation -- by keeping its scratch in a fixed
device array.  Two calls in a row (different matrices, both reference forms)
must match the planned SpMV within the FP64 tolerance of the other SpMV tests
(1e-13 relative 2-norm); since both run the same kernels they are in fact
bit-identical.  This file is collected last on purpose.
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


def test_noalloc_spmv_matches_planned_spmv_twice(lab):
    from linearalgebra_b200 import gen
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
