"""Adjoint gradients through the wave-equation operator in PROPAG's own form
with node coefficients (MATDIFUV with u = DM1 and v = HPROP, the depth; and
MATDIF with u per node): autograd's dL/du and dL/dv against an exact dense
binary64 reference built from the oracle's assembly, and against centred
finite differences of the device solve."""
import numpy as np
import pytest

from opentelemac_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _dense(oracle_mod, x, y, ik, u, v, kind, xmm, xmd):
    dm, xm = oracle_mod.mass_diff_matrix(x, y, ik, u, v, kind=kind, xmul_mass=xmm, xmul_dif=xmd)
    n = x.size
    eye = np.eye(n)
    return np.stack([oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", eye[:, j])
                     for j in range(n)], axis=1)


def _fields(n, kind, seed, h):
    """Node coefficients scaled as PROPAG's are: DM1 = -TETAU TETAH GRAV
    V2DPAR / (1/DT + FROT) carries the nodal area (~h^2), so the mass and
    diffusion terms stay comparable on any mesh (condition number ~1e3-1e4
    here); u for MATDIF likewise."""
    rng = np.random.default_rng(seed)
    if kind == 11:
        return h * h * rng.uniform(5.0, 50.0, n), None, 1.0, 1.0
    dm1 = -9.81 * h * h * rng.uniform(0.5, 2.0, n)
    hprop = rng.uniform(1.0, 50.0, n)
    return dm1, hprop, 1.0, -1.0


@pytest.mark.parametrize("kind", [11, 12])
def test_node_coefficient_gradient_vs_dense(oracle_mod, kind):
    import torch
    from opentelemac_b200.autograd import MassDiffProblem, mass_diff_solve
    x, y, ik = mg.square_mesh(11)
    x, y, ik, _, _ = mg.shuffled(x, y, ik)
    n = x.size
    u, v, xmm, xmd = _fields(n, kind, 3, 0.1)
    rng = np.random.default_rng(4)
    b = rng.uniform(-1, 1, n)
    xobs = rng.uniform(-1, 1, n)
    # dense reference: A is linear in u (v fixed) and in v (u fixed), so
    # dA/du_i = A(u + e_i) - A(u) exactly up to rounding
    A0 = _dense(oracle_mod, x, y, ik, u, v, kind, xmm, xmd)
    xs = np.linalg.solve(A0, b)
    lam = np.linalg.solve(A0.T, xs - xobs)     # L = 0.5 |x - xobs|^2
    gu_ref = np.empty(n)
    gv_ref = np.empty(n) if kind == 12 else None
    for i in range(n):
        du = u.copy()
        du[i] += 1.0
        gu_ref[i] = -lam @ (_dense(oracle_mod, x, y, ik, du, v, kind, xmm, xmd) - A0) @ xs
        if kind == 12:
            dv = v.copy()
            dv[i] += 1.0
            gv_ref[i] = -lam @ (_dense(oracle_mod, x, y, ik, u, dv, kind, xmm, xmd) - A0) @ xs
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    prob = MassDiffProblem(x, y, ik, kind=kind, xmul_mass=xmm, xmul_dif=xmd)
    ut = t(u).requires_grad_(True)
    vt = t(v).requires_grad_(True) if kind == 12 else None
    bt = t(b).requires_grad_(True)
    xt = mass_diff_solve(ut, vt, bt, prob)
    np.testing.assert_allclose(xt.detach().cpu().numpy(), xs, rtol=1e-8,
                               atol=1e-10 * np.abs(xs).max())
    loss = 0.5 * ((xt - t(xobs)) ** 2).sum()
    loss.backward()
    # the dense route -lam^T (A(u+e_i) - A(u)) x cancels the solution's large
    # smooth components through row sums that are zero only up to rounding:
    # its own error is ~3e-9 of the largest entry (checked in extended
    # precision), hence the absolute tolerance
    scale = np.abs(gu_ref).max()
    np.testing.assert_allclose(ut.grad.cpu().numpy(), gu_ref, rtol=1e-7, atol=1e-8 * scale)
    np.testing.assert_allclose(bt.grad.cpu().numpy(), lam, rtol=1e-7,
                               atol=1e-9 * np.abs(lam).max())
    if kind == 12:
        scale = np.abs(gv_ref).max()
        np.testing.assert_allclose(vt.grad.cpu().numpy(), gv_ref, rtol=1e-7, atol=1e-8 * scale)
    prob.close()


def test_depth_gradient_vs_finite_differences():
    """dL/dHPROP on a 101 x 101 mesh with L = 0.5 |x(v) - x(v0)|^2, v = v0 +
    noise: 32 random nodes against centred differences of the device solve
    with a step of 1e-4 of the node's depth (the truncation error of that
    step, measured with direct sparse solves, stays below 1e-6), median
    relative error and a directional derivative through all 32 below 1e-5."""
    import torch
    from opentelemac_b200.autograd import MassDiffProblem, mass_diff_solve
    x, y, ik = mg.square_mesh(101)
    n = x.size
    u, v0, xmm, xmd = _fields(n, 12, 5, 0.01)
    rng = np.random.default_rng(6)
    v = v0 * (1.0 + 0.05 * rng.standard_normal(n))
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    prob = MassDiffProblem(x, y, ik, kind=12, xmul_mass=xmm, xmul_dif=xmd, eps=1e-14)
    ut, b = t(u), t(rng.uniform(-1, 1, n))
    with torch.no_grad():
        xobs = mass_diff_solve(ut, t(v0), b, prob)
    loss = lambda vv: 0.5 * ((mass_diff_solve(ut, vv, b, prob) - xobs) ** 2).sum()
    vt = t(v).requires_grad_(True)
    loss(vt).backward()
    g = vt.grad.cpu().numpy()
    picks = rng.choice(n, 32, replace=False)
    rel = []
    with torch.no_grad():
        for i in picks:
            h = 1e-4 * v[i]
            vp, vm = v.copy(), v.copy()
            vp[i] += h
            vm[i] -= h
            fd = (float(loss(t(vp))) - float(loss(t(vm)))) / (2 * h)
            rel.append(abs(fd - g[i]) / abs(g[i]))
        d = np.zeros(n)
        d[picks] = rng.uniform(-1, 1, 32) * 1e-4 * v[picks]
        fdd = float(loss(t(v + d))) - float(loss(t(v - d)))
    gd = 2 * float(g @ d)
    assert np.median(rel) < 1e-5, np.median(rel)
    assert abs(fdd - gd) / abs(gd) < 1e-5, (fdd, gd)
    prob.close()
