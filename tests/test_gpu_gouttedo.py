"""The device path on the reference's own mesh: gouttedo (TELEMAC-2D example
`examples/telemac2d/gouttedo`, 4,624 nodes and 8,978 triangles in the
reference's node and element numbering, frozen in tests/golden/gouttedo.npz).

The operator is PROPAG's wave-equation matrix at the case's first time step
(MATMAS/DT + MATDIFUV, DT 0.04, implicitation 0.6, the drop's initial
depth), assembled on the device.  Checked bit for bit against the oracle:
the assembly, every MATVEC operation, and SOLVE with the case's own settings
(t2d_gouttedo_reprod.cas: SOLVER 1, PRECONDITIONING 0, SOLVER ACCURACY 1e-4,
100 iterations, FINITE ELEMENT ASSEMBLY 3 -- compensated dot products) in
the reference's sequential summation order, then the same to convergence
with diagonal preconditioning, in segment storage, and the mixed solve."""
import numpy as np
import pytest

from conftest import GOUTTEDO_DT, gouttedo_problem
from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu
OPS = ["X=AY    ", "X=X+AY  ", "X=-AY   ", "X=X-AY  ", "X=X+CAY ", "X=CAY   ",
       "X=TAY   ", "X=-TAY  ", "X=X+TAY ", "X=X-TAY ", "X=X+CTAY"]


@pytest.fixture(scope="module")
def gd(oracle_mod):
    return gouttedo_problem(oracle_mod)


def _device_matrix(p):
    import torch
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    mesh = bief.Mesh(p["ik"], p["x"].size)
    A = bief.Matrix(mesh)
    A.assemble_mass_diff(t(p["x"]), t(p["y"]), t(p["dm1"]), t(p["h"]), kind=12,
                         xmul_mass=1.0 / GOUTTEDO_DT, xmul_dif=-1.0)
    return mesh, A


def test_gouttedo_assembly_and_matvec(oracle_mod, gd):
    mesh, A = _device_matrix(gd)
    dm, xm, td = A.get()
    assert td == "Q"
    assert np.array_equal(dm, gd["dm"]) and np.array_equal(xm, gd["xm"])
    rng = np.random.default_rng(11)
    y = rng.uniform(-1, 1, dm.size)
    x0 = rng.uniform(-1, 1, dm.size)
    for op in OPS:
        got = x0.copy()
        bief.matvec(op, got, A, y, c=0.7)
        ref = oracle_mod.matvec(op, gd["ik"], gd["dm"], "Q", gd["xm"], "S", y, c=0.7, x=x0)
        np.testing.assert_array_equal(got, ref, err_msg=op)
    mesh.close()


@pytest.mark.parametrize("precon,eps,nitmax", [(0, 1e-4, 100), (2, 1e-12, 100000)])
def test_gouttedo_modass3_reference_order(oracle_mod, gd, precon, eps, nitmax):
    """MODASS = 3: the device's compensated GRACJG equals the restatement
    run in the reference's own sequential order (DOT_COMP), every bit of X,
    the iteration count and the residual -- first with the case's own
    solver settings, then converged with diagonal preconditioning."""
    mesh, A = _device_matrix(gd)
    n = gd["x"].size
    cfg = bief.SlvCfg(slv=1, nitmax=nitmax, precon=precon, krylov=0, eps=eps, zero=0.0)
    x = np.zeros(n)
    b = gd["b"].copy()
    st, nit, relres = bief.solve(x, A, b, cfg, modass=3, mutate=True)
    dm_out, xm_out, td = A.get()
    r = oracle_mod.solve(gd["ik"], gd["dm"], "Q", gd["xm"], "S", gd["b"], precon=precon,
                         eps=eps, nitmax=nitmax, dot_mode=oracle_mod.DOT_COMP_SEQUENTIAL)
    assert st == r["status"] and nit == r["nit"] and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    # SOLVE's side effects (none for PRECONDITIONING 0, which SOLVE makes 1)
    np.testing.assert_array_equal(b, r["b"])
    np.testing.assert_array_equal(dm_out, r["dm"])
    np.testing.assert_array_equal(xm_out, r["xm"])
    assert td == r["typdia"]
    mesh.close()


def test_gouttedo_modass1_device_order_and_reference_order(oracle_mod, gd):
    """MODASS = 1: bit for bit in the device's dot order; in the reference's
    sequential order the converged solutions agree to 1e-10."""
    mesh, A = _device_matrix(gd)
    n = gd["x"].size
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-13, zero=0.0)
    x = np.zeros(n)
    st, nit, relres = bief.solve(x, A, gd["b"].copy(), cfg)
    G, T = mesh.launch_info()
    r = oracle_mod.solve(gd["ik"], gd["dm"], "Q", gd["xm"], "S", gd["b"], eps=1e-13,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == r["status"] == 0 and nit == r["nit"] and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    s = oracle_mod.solve(gd["ik"], gd["dm"], "Q", gd["xm"], "S", gd["b"], eps=1e-13)
    assert s["status"] == 0
    assert np.linalg.norm(x - s["x"]) <= 1e-10 * np.linalg.norm(s["x"])
    mesh.close()


def test_gouttedo_segments_and_mixed(oracle_mod, gd):
    """Segment storage (the TELEMAC-2D default) with STOSEG's numbering of
    the gouttedo mesh, and the mixed-precision solve: bit for bit."""
    mesh, A = _device_matrix(gd)
    n = gd["x"].size
    G, T = mesh.launch_info()
    x = np.zeros(n)
    st, outer, inner, relres = bief.solve_mixed(x, A, gd["b"], precon=2, inner_tol=0.1,
                                                outer_tol=1e-10)
    r = oracle_mod.solve_mixed(gd["ik"], gd["dm"], "Q", gd["xm"], gd["b"], precon=2,
                               inner_tol=0.1, outer_tol=1e-10, max_outer=1000,
                               max_inner=1000000, nblocks=G, nthreads=T)
    assert st == r["status"] == 0 and (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])

    g1, g2, es, ori = mg.segments(gd["ik"], n)
    mesh.set_segments(g1, g2)
    A.to_segments()
    xa = oracle_mod.assex3(es, ori, "S", gd["xm"], g1.size)
    x = np.zeros(n)
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-12, zero=0.0)
    st, nit, relres = bief.solve(x, A, gd["b"].copy(), cfg, modass=3)
    r = oracle_mod.solve_seg(g1, g2, gd["dm"], "Q", xa, "S", gd["b"], eps=1e-12,
                             dot_mode=oracle_mod.DOT_COMP_SEQUENTIAL)
    assert st == r["status"] == 0 and nit == r["nit"] and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    mesh.close()
