"""Adjoint gradients (no reference counterpart: the reference has none).

* torch.autograd.gradcheck of the SpMV and of the full IC(0)-PCG solve on
  small SPD stencils (the solve parameterised by its upper triangle, so
  perturbations keep A symmetric and CG valid);
* the differentiation configuration at full size -- SPD 27-point stencil on a
  96^3 grid, off-diagonals -U[0.5, 1.5], diagonal 1.05 x row abs-sum, FP64;
  L = 1/2 ||u - u*||^2 with u = A^-1 b, u*, b ~ N(0, 1): the adjoint dL/db and
  dL/dvalues, and the SpMV adjoint (dL/dx, dL/dvalues) for
  L = 1/2 ||A x - y*||^2, each checked by central finite differences on 64
  random entries (<= 1e-6 relative) and against an FP64 CPU gradient from the
  oracle.
Finite differences (central; fourth order for the matrix values, in which L
is not quadratic) form each L(+h) - L(-h) from the two solutions directly,
sum_i (u+_i - u-_i) (0.5 (u+_i + u-_i) - u*_i), so the large constant part of
L does not cancel in floating point.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dtype)


def _solver(lab, n, ai, aj, av):
    from linearalgebra_b200 import gen
    ua, uj, uv = gen.upper_with_diag(n, ai, aj, av)
    f = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    A = lab.CSR(n, n, 0, ai, aj, av)
    return lab.PCG(A, ua, uj, f), uv


def test_gradcheck_solve_and_spmv_small(lab):
    from linearalgebra_b200 import autograd as lag
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.stencil27(4, seed=7)
    solver, uv = _solver(lab, n, ai, aj, av)
    f = lag.SymmetricSolve(solver, n, ai, aj, rtol=1e-14)
    upper = _dev(uv).requires_grad_(True)
    b = _dev(np.random.default_rng(1).standard_normal(n)).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda v, bb: f(v, bb), (upper, b), eps=1e-6,
                                    atol=1e-8, rtol=1e-5)
    plan = lab.SPMV(lab.CSR(n, n, 0, ai, aj, av))
    vals = _dev(av).requires_grad_(True)
    x = _dev(np.random.default_rng(2).standard_normal(n)).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda v, xx: lag.spmv(plan, v, xx), (vals, x),
                                    eps=1e-6, atol=1e-8, rtol=1e-6)


def _dl(up, um, target):
    return float(torch.dot(up - um, 0.5 * (up + um) - target))


def test_differentiation_config_full_size(lab, orc):
    from linearalgebra_b200 import autograd as lag
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.stencil27(96, seed=0)
    assert n == 884_736 and int(ai[-1]) == 23_393_656
    rng = np.random.default_rng(0)
    ustar = rng.standard_normal(n)
    bvec = rng.standard_normal(n)
    solver, uv = _solver(lab, n, ai, aj, av)
    f = lag.SymmetricSolve(solver, n, ai, aj, rtol=1e-14)
    idx = f.index
    upper = _dev(uv).requires_grad_(True)
    b = _dev(bvec).requires_grad_(True)
    us = _dev(ustar)
    u = f(upper, b)
    L = 0.5 * torch.sum((u - us) ** 2)
    L.backward()
    g_up, g_b = upper.grad.detach().clone(), b.grad.detach().clone()
    u0 = u.detach().clone()

    def solve(upper_vals, bb):
        with torch.no_grad():
            return f(upper_vals, bb)

    # dL/db by central differences on 64 random entries; relative errors use
    # max(|g|, 1e-3 * rms(g)) so that a near-zero entry cannot blow up
    floor = float(torch.sqrt(torch.mean(g_b ** 2)))
    ks = rng.choice(n, 64, replace=False)
    worst = 0.0
    for k in ks:
        h = 1e-3
        bp, bm = b.detach().clone(), b.detach().clone()
        bp[k] += h
        bm[k] -= h
        fd = _dl(solve(upper.detach(), bp), solve(upper.detach(), bm), us) / (2 * h)
        g = float(g_b[k])
        worst = max(worst, abs(fd - g) / max(abs(g), 1e-3 * floor))
    print(f"dL/db: worst FD relative error over 64 entries {worst:.2e}")
    assert worst <= 1e-6
    # dL/dvalues (upper-triangle parameters; off-diagonal ones move a_ij and a_ji)
    nup = len(uv)
    floor = float(torch.sqrt(torch.mean(g_up ** 2)))
    ks = rng.choice(nup, 64, replace=False)
    worst = 0.0
    def at(k, d):
        v = upper.detach().clone()
        v[k] += d
        return solve(v, b.detach())

    for k in ks:
        # L is not quadratic in the matrix values: fourth-order central
        # difference (8 [L(+h) - L(-h)] - [L(+2h) - L(-2h)]) / 12h
        h = 1e-3 * max(1.0, abs(uv[k]))
        d1 = _dl(at(k, h), at(k, -h), us)
        d2 = _dl(at(k, 2 * h), at(k, -2 * h), us)
        fd = (8 * d1 - d2) / (12 * h)
        g = float(g_up[k])
        worst = max(worst, abs(fd - g) / max(abs(g), 1e-3 * floor))
    print(f"dL/dvalues: worst FD relative error over 64 entries {worst:.2e}")
    assert worst <= 1e-6

    # FP64 CPU gradient from the oracle: u = A^-1 b, lambda = A^-1 (u - u*),
    # dL/db = lambda, dL/dA_ij = -lambda_i u_j (mirrored pairs added)
    P = orc.ptr
    ua, uj, _ = gen.upper_with_diag(n, ai, aj, av)
    fac = lab.ICCLevelNumeric0(n, 0, ua, uj, uv)
    u_cpu = np.zeros(n)
    lam = np.zeros(n)
    r = np.zeros(1)
    assert orc.port().oracle_pcg(n, 0, P(ai), P(aj), P(av), P(ua), P(uj), P(fac), P(bvec),
                                 P(u_cpu), 1e-13, 2000, P(r)) > 0
    rhs = u_cpu - ustar
    assert orc.port().oracle_pcg(n, 0, P(ai), P(aj), P(av), P(ua), P(uj), P(fac), P(rhs),
                                 P(lam), 1e-13, 2000, P(r)) > 0
    rows = np.repeat(np.arange(n), np.diff(ai))
    g_full = -lam[rows] * u_cpu[aj]
    g_up_cpu = np.zeros(nup)
    np.add.at(g_up_cpu, idx.cpu().numpy(), g_full)
    e_b = np.linalg.norm(g_b.cpu().numpy() - lam) / np.linalg.norm(lam)
    e_v = np.linalg.norm(g_up.cpu().numpy() - g_up_cpu) / np.linalg.norm(g_up_cpu)
    e_u = np.linalg.norm(u0.cpu().numpy() - u_cpu) / np.linalg.norm(u_cpu)
    print(f"vs FP64 CPU gradient: u {e_u:.2e}, dL/db {e_b:.2e}, dL/dvalues {e_v:.2e}")
    assert e_u <= 1e-9 and e_b <= 1e-9 and e_v <= 1e-9

    # SpMV adjoint on the same matrix: L = 1/2 ||A x - y*||^2
    plan = lab.SPMV(lab.CSR(n, n, 0, ai, aj, av))
    vals = _dev(av).requires_grad_(True)
    x = _dev(rng.standard_normal(n)).requires_grad_(True)
    ys = _dev(rng.standard_normal(n))
    y = lag.spmv(plan, vals, x)
    (0.5 * torch.sum((y - ys) ** 2)).backward()
    gx, gv = x.grad.detach(), vals.grad.detach()
    fx, fv = float(torch.sqrt(torch.mean(gx ** 2))), float(torch.sqrt(torch.mean(gv ** 2)))
    worst = 0.0
    for k in rng.choice(n, 64, replace=False):
        h = 1e-3
        xp, xm = x.detach().clone(), x.detach().clone()
        xp[k] += h
        xm[k] -= h
        with torch.no_grad():
            fd = _dl(lag.spmv(plan, vals.detach(), xp), lag.spmv(plan, vals.detach(), xm), ys)
        fd /= 2 * h
        worst = max(worst, abs(fd - float(gx[k])) / max(abs(float(gx[k])), 1e-3 * fx))
    for k in rng.choice(len(av), 64, replace=False):
        h = 1e-3
        vp, vm = vals.detach().clone(), vals.detach().clone()
        vp[k] += h
        vm[k] -= h
        with torch.no_grad():
            fd = _dl(lag.spmv(plan, vp, x.detach()), lag.spmv(plan, vm, x.detach()), ys)
        fd /= 2 * h
        worst = max(worst, abs(fd - float(gv[k])) / max(abs(float(gv[k])), 1e-3 * fv))
    print(f"SpMV adjoint: worst FD relative error over 128 entries {worst:.2e}")
    assert worst <= 1e-6
    # against the FP64 CPU gradient
    xn = x.detach().cpu().numpy()
    yv = np.zeros(n)
    orc.port().oracle_serial_spmv(n, 0, P(ai), P(aj), P(av), P(xn), P(yv), 1.0, 0.0)
    res = yv - ys.cpu().numpy()
    gx_cpu = np.zeros(n)
    orc.port().oracle_spmv_transpose(n, n, 0, P(ai), P(aj), P(av), P(res), P(gx_cpu), 1.0, 0.0)
    gv_cpu = res[rows] * xn[aj]
    assert np.linalg.norm(gx.cpu().numpy() - gx_cpu) <= 1e-12 * np.linalg.norm(gx_cpu)
    assert np.linalg.norm(gv.cpu().numpy() - gv_cpu) <= 1e-12 * np.linalg.norm(gv_cpu)
