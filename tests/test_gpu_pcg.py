"""GPU IC(0)-PCG (FP64 and mixed) vs the oracle's FP64 PCG.

Both stop on the true FP64 residual ||b - A x|| / ||b|| < 1e-10; the
iteration counts agree with the oracle's within 2 (different but valid
summation orders), the FP64 solutions agree to 1e-8, and the mixed result
states its error against the FP64 solution.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", torch.float64)


def setup(lab, n, ai, aj, av):
    from linearalgebra_b200 import gen
    iperm, perm = lab.SerialCM(n, 0, ai, aj)
    b_ai, b_aj, b_av = lab.Permute(n, 0, ai, aj, av, iperm, perm)
    ua, uj, uv = gen.upper_with_diag(n, b_ai, b_aj, b_av)
    f = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    return (b_ai, b_aj, b_av), (ua, uj, f)


@pytest.mark.parametrize("case", ["lap3d_24", "st27_16", "aniso_20"])
def test_pcg_fp64_and_mixed(lab, orc, case):
    from linearalgebra_b200 import gen
    n, ai, aj, av = {"lap3d_24": lambda: gen.laplacian_3d(24),
                     "st27_16": lambda: gen.stencil27(16),
                     "aniso_20": lambda: gen.aniso7(20, seed=2)}[case]()
    (b_ai, b_aj, b_av), (ua, uj, f) = setup(lab, n, ai, aj, av)
    b = np.random.default_rng(0).uniform(-1, 1, n)
    P = orc.ptr
    xo = np.zeros(n)
    ro = np.zeros(1)
    it_o = orc.port().oracle_pcg(n, 0, P(b_ai), P(b_aj), P(b_av), P(ua), P(uj), P(f), P(b),
                                 P(xo), 1e-10, 20000, P(ro))
    assert it_o > 0
    A = lab.CSR(n, n, 0, b_ai, b_aj, b_av, keep_f32=True)
    s = lab.PCG(A, ua, uj, f)
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    r = s.solve(dev(b), x, rtol=1e-10, maxit=20000)
    xn = x.cpu().numpy()
    true_rel = np.linalg.norm(b - _spmv_np(b_ai, b_aj, b_av, xn)) / np.linalg.norm(b)
    assert r.rel_residual < 1e-10 and true_rel < 1e-10
    assert abs(r.iterations - it_o) <= 2, (r.iterations, it_o)
    assert np.linalg.norm(xn - xo) <= 1e-8 * np.linalg.norm(xo)
    m = lab.PCG(A, ua, uj, f, mixed=True)
    xm = torch.empty(n, dtype=torch.float64, device="cuda")
    rm = m.solve(dev(b), xm, rtol=1e-10, maxit=20000)
    xmn = xm.cpu().numpy()
    true_m = np.linalg.norm(b - _spmv_np(b_ai, b_aj, b_av, xmn)) / np.linalg.norm(b)
    err = np.linalg.norm(xmn - xo) / np.linalg.norm(xo)
    print(f"{case}: fp64 {r.iterations} it, mixed {rm.iterations} inner / "
          f"{rm.outer_iterations} outer, mixed resid {true_m:.2e}, err vs fp64 {err:.2e}")
    assert rm.rel_residual < 1e-10 and true_m < 1e-10
    assert err < 1e-7


def _spmv_np(ai, aj, av, x):
    rows = np.repeat(np.arange(len(ai) - 1), np.diff(ai))
    return np.bincount(rows, weights=av * x[aj], minlength=len(ai) - 1)


def test_pcg_host_path_and_not_converged(lab):
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_2d(48)
    (b_ai, b_aj, b_av), (ua, uj, f) = setup(lab, n, ai, aj, av)
    A = lab.CSR(n, n, 0, b_ai, b_aj, b_av)
    s = lab.PCG(A, ua, uj, f)
    b = np.random.default_rng(1).uniform(-1, 1, n)
    x = np.zeros(n)
    r = s.solve(b, x, rtol=1e-10)
    assert r.rel_residual < 1e-10
    r2 = s.solve(b, x, rtol=1e-10, maxit=3, allow_not_converged=True)
    assert r2.status == "LA_ERR_NOT_CONVERGED" and r2.iterations == 3
    with pytest.raises(lab.LAError):
        s.solve(b, x, rtol=1e-10, maxit=3)


@pytest.mark.parametrize("case", ["lap3d_32", "aniso_24"])
def test_pcg_fused_iteration_bit_identical(lab, monkeypatch, case):
    """The fused iteration (dot products finished inside two cooperative
    vector kernels, the solves' sentinel written by the update) gives the
    same iterates as the separate dot / update launches, bit for bit, in FP64
    and mixed precision: same iteration counts, same x."""
    from linearalgebra_b200 import gen
    n, ai, aj, av = {"lap3d_32": lambda: gen.laplacian_3d(32),
                     "aniso_24": lambda: gen.aniso7(24, seed=4)}[case]()
    (b_ai, b_aj, b_av), (ua, uj, f) = setup(lab, n, ai, aj, av)
    A = lab.CSR(n, n, 0, b_ai, b_aj, b_av, keep_f32=True)
    b = dev(np.random.default_rng(7).uniform(-1, 1, n))
    for mixed in (False, True):
        monkeypatch.setenv("LA_PCG_FUSED", "0")
        s0 = lab.PCG(A, ua, uj, f, mixed=mixed)
        monkeypatch.delenv("LA_PCG_FUSED")
        s1 = lab.PCG(A, ua, uj, f, mixed=mixed)
        assert not s0.fused() and s1.fused()
        x0 = torch.empty(n, dtype=torch.float64, device="cuda")
        x1 = torch.empty_like(x0)
        r0 = s0.solve(b, x0, rtol=1e-10, maxit=20000)
        r1 = s1.solve(b, x1, rtol=1e-10, maxit=20000)
        assert (r0.iterations, r0.outer_iterations) == (r1.iterations, r1.outer_iterations)
        assert torch.equal(x0, x1), (case, mixed)
        assert r1.rel_residual == r0.rel_residual
        print(f"{case} mixed={mixed}: {r1.iterations} it, fused {r1.solve_ms:.2f} ms, "
              f"unfused {r0.solve_ms:.2f} ms")
