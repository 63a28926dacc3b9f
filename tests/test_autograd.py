"""Adjoint gradient of the wave solve (torch.autograd.Function whose backward
runs the adjoint CG on the library kernels) against centred finite
differences, a dense binary64 gradient, and the checkpointed unrolled loop
against the plain one."""
import numpy as np
import pytest

from opentelemac_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _setup(n, seed=3, eps=1e-13):
    import torch
    from opentelemac_b200 import autograd as ag
    x, y, ik = mg.square_mesh(n)
    prob = ag.WaveProblem(x, y, ik, eps=eps)
    h0 = torch.tensor(mg.depth_smooth(x, y, ik), device="cuda")
    rng = np.random.default_rng(seed)
    h = h0 + torch.tensor(rng.normal(0.0, 0.1, ik.shape[0]), device="cuda")
    xt = torch.tensor(mg.random_solution(x.size), device="cuda")
    A0 = prob.assemble(mg.DT * mg.GRAV * h0)
    b = torch.zeros_like(xt)
    from opentelemac_b200 import bief
    bief.matvec("X=AY    ", b, A0, xt)
    x_obs = prob.solve(mg.DT * mg.GRAV * h0, b)
    return prob, x, y, ik, h0, h, b, x_obs


def _loss(prob, h, b, x_obs):
    from opentelemac_b200 import autograd as ag
    x = ag.wave_solve(mg.DT * mg.GRAV * h, b, prob)
    return 0.5 * ((x - x_obs) ** 2).sum()


def test_adjoint_gradient_vs_finite_differences_501():
    """501 x 501 nodes (251,001 nodes, 500,000 triangles): dL/dh on 64
    random elements against centred differences.  With eps = 1e-3 (relative
    2e-4 of h) the agreement is 1e-6 per element and along a direction.
    With eps = 1e-6 on a single element the difference L(h+) - L(h-) is
    ~1e-10 of L and the comparison is bounded by the binary64 rounding of L
    and of the two solves (measured 3e-4 per element, 5e-5 along a
    direction through all 64), which the test records."""
    import torch
    prob, x, y, ik, h0, h, b, x_obs = _setup(501)
    hv = h.clone().requires_grad_(True)
    L = _loss(prob, hv, b, x_obs)
    L.backward()
    g = hv.grad
    rng = np.random.default_rng(11)
    picks = rng.choice(ik.shape[0], 64, replace=False)
    ga = g[torch.tensor(picks, device="cuda")].cpu().numpy()
    v = torch.zeros_like(h)
    v[torch.tensor(picks, device="cuda")] = torch.tensor(rng.uniform(-1, 1, 64), device="cuda")
    gv = (g * v).sum().item()

    def fd_checks(eps):
        fd = []
        with torch.no_grad():
            for e in picks:
                hp, hm = h.clone(), h.clone()
                hp[e] += eps
                hm[e] -= eps
                fd.append(((_loss(prob, hp, b, x_obs) - _loss(prob, hm, b, x_obs)) / (2 * eps)).item())
            d = ((_loss(prob, h + eps * v, b, x_obs) - _loss(prob, h - eps * v, b, x_obs)) / (2 * eps)).item()
        rel = np.abs(np.array(fd) - ga) / np.abs(ga)
        return np.median(rel), abs(d - gv) / abs(gv)

    med, drel = fd_checks(1e-3)
    assert med < 1e-6 and drel < 1e-6
    med, drel = fd_checks(1e-6)
    assert med < 2e-3 and drel < 5e-4
    prob.close()


def test_adjoint_gradient_vs_dense_21():
    """21 x 21 nodes: the gradient against a dense binary64 computation
    (numpy element matrices, numpy.linalg.solve)."""
    import torch
    prob, x, y, ik, h0, h, b, x_obs = _setup(21)
    hv = h.clone().requires_grad_(True)
    L = _loss(prob, hv, b, x_obs)
    L.backward()
    g = hv.grad.cpu().numpy()
    # dense reference
    X, Y = x[ik], y[ik]
    bb = Y[:, [1, 2, 0]] - Y[:, [2, 0, 1]]
    cc = X[:, [2, 0, 1]] - X[:, [1, 2, 0]]
    area = 0.5 * ((X[:, 1] - X[:, 0]) * (Y[:, 2] - Y[:, 0]) - (X[:, 2] - X[:, 0]) * (Y[:, 1] - Y[:, 0]))
    K = (bb[:, :, None] * bb[:, None, :] + cc[:, :, None] * cc[:, None, :]) / (4 * area)[:, None, None]
    M = area[:, None, None] / 12.0 * (np.ones((3, 3)) + np.eye(3))
    coef = mg.DT * mg.GRAV * h.cpu().numpy()
    n = x.size
    A = np.zeros((n, n))
    for e in range(ik.shape[0]):
        A[np.ix_(ik[e], ik[e])] += M[e] + coef[e] * K[e]
    xs = np.linalg.solve(A, b.cpu().numpy())
    lam = np.linalg.solve(A, xs - x_obs.cpu().numpy())
    gref = -mg.DT * mg.GRAV * np.einsum("ei,eij,ej->e", lam[ik], K, xs[ik])
    np.testing.assert_allclose(g, gref, rtol=1e-7, atol=1e-9 * np.abs(gref).max())
    assert abs(L.item() - 0.5 * np.sum((xs - x_obs.cpu().numpy()) ** 2)) <= 1e-9 * max(L.item(), 1e-30)
    prob.close()


def test_unrolled_loop_checkpointing():
    """50 implicit steps x_{n+1} = A^-1 M x_n: the loop that keeps one state
    in ten (recomputing the rest in backward) gives the same gradient bits
    as the loop that keeps all states, and matches finite differences."""
    import torch
    from opentelemac_b200 import autograd as ag
    prob, x, y, ik, h0, h, b, x_obs = _setup(51)
    # a smooth initial state and a small time step (dt = 1e-4), so that 50
    # implicit steps still carry information about h
    x0 = torch.tensor(np.sin(np.pi * x) * np.cos(2 * np.pi * y), device="cuda")
    dtg = 1e-4 * mg.GRAV
    with torch.no_grad():
        target = ag.unrolled_loop(dtg * h0, x0, prob, nsteps=50, checkpoint_every=0)

    def run(ck):
        hv = h.clone().requires_grad_(True)
        xn = ag.unrolled_loop(dtg * hv, x0, prob, nsteps=50, checkpoint_every=ck)
        L = 0.5 * ((xn - target) ** 2).sum()
        s0 = prob.solves
        L.backward()
        return L.item(), hv.grad.clone(), prob.solves - s0

    L1, g1, nsolve_ck = run(10)
    L2, g2, nsolve_plain = run(0)
    assert L1 == L2
    assert torch.equal(g1, g2)
    assert nsolve_ck == 100 and nsolve_plain == 50   # recomputed forward + adjoint
    rng = np.random.default_rng(2)
    v = torch.tensor(rng.uniform(-1, 1, ik.shape[0]), device="cuda")
    eps = 1e-3
    with torch.no_grad():
        def lossv(hh):
            xn = ag.unrolled_loop(dtg * hh, x0, prob, nsteps=50, checkpoint_every=10)
            return 0.5 * ((xn - target) ** 2).sum().item()
        d = (lossv(h + eps * v) - lossv(h - eps * v)) / (2 * eps)
    gv = (g1 * v).sum().item()
    assert abs(gv) > 1e-8
    assert abs(d - gv) <= 1e-5 * abs(gv)
    prob.close()
