"""Full-size workloads checked through size-independent properties.

The 1001 x 1001 smooth-depth solve (1,002,001 nodes, relres 1e-8) and the
2001 x 2001 log-uniform-depth solve (4,004,001 nodes, refinement to relres
1e-10 with a binary32 inner CG) are too large for the oracle, so each is
checked by:
  - the returned relres equals an independently computed scaled residual
    ||D (b - A x)|| / ||D b|| (D = 1/sqrt(DM), PRECON = 2), within rounding;
  - both solvers converge, and the mixed solve's iteration count stays near
    the binary64 one;
  - the mixed solution's distance from the binary64 solution is reported and
    bounded.
"""
import numpy as np
import pytest

from opentelemac_b200 import bief, meshgen as mg


def _setup(n, depth):
    import torch
    x, y, ik = mg.square_mesh(n)
    h = mg.depth_loguniform(ik) if depth == "loguniform" else mg.depth_smooth(x, y, ik)
    mesh = bief.Mesh(ik, x.size)
    A = bief.Matrix(mesh)
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    A.assemble_wave(t(x), t(y), t(mg.wave_coef(h)))
    xt = t(mg.random_solution(x.size))
    b = torch.zeros_like(xt)
    bief.matvec("X=AY    ", b, A, xt)
    return mesh, A, b, xt


def _scaled_relres(A, b, x):
    import torch
    r = torch.empty_like(b)
    bief.matvec("X=AY    ", r, A, x)
    r = b - r
    dm = torch.tensor(A.get()[0], device=b.device)
    d = 1.0 / torch.sqrt(dm)
    return float(torch.linalg.norm(d * r) / torch.linalg.norm(d * b))


@pytest.mark.gpu
@pytest.mark.parametrize("n,depth,eps,itol,err_max", [
    (1001, "smooth", 1e-8, 0.1, 1e-6),
    (2001, "loguniform", 1e-10, 1e-4, 2e-5),
    (2001, "loguniform", 1e-10, 0.1, 2e-5),
])
def test_full_size_mixed_vs_fp64(n, depth, eps, itol, err_max):
    import torch
    mesh, A, b, xt = _setup(n, depth)
    x64 = torch.zeros_like(b)
    cfg = bief.SlvCfg(slv=1, nitmax=1000000, precon=2, krylov=0, eps=eps, zero=0.0)
    st, nit64, rel64 = bief.solve(x64, A, b, cfg)
    assert st == 0 and rel64 <= eps
    assert _scaled_relres(A, b, x64) == pytest.approx(rel64, rel=1e-3)

    xm = torch.zeros_like(b)
    st, outer, inner, relm = bief.solve_mixed(xm, A, b, precon=2, inner_tol=itol, outer_tol=eps)
    assert st == 0 and relm <= eps
    # the returned relres is the binary64 residual of the returned solution
    assert _scaled_relres(A, b, xm) == pytest.approx(relm, rel=1e-3)
    assert inner <= 1.25 * nit64
    err = float(torch.linalg.norm(xm - x64) / torch.linalg.norm(x64))
    assert err <= err_max
    # both are equally far from the manufactured solution (the residual, not
    # the precision, bounds the error)
    e64 = float(torch.linalg.norm(x64 - xt) / torch.linalg.norm(xt))
    em = float(torch.linalg.norm(xm - xt) / torch.linalg.norm(xt))
    assert em == pytest.approx(e64, rel=1e-2)
    mesh.close()
