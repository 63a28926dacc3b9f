"""The persistent solvers in both residencies (one or two blocks per SM,
bief_set_blocks_per_sm): every SOLVE method and the mixed-precision solve,
bit for bit against the oracle run in the dot-product tree the launch
reports (bief_launch_info)."""
import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu

# SLV: 1 CG, 2 conjugate residual, 3 CG on the normal equations, 4 minimum
# error, 5 squared CG, 6 CGSTAB, 7 GMRES
METHODS = [1, 2, 3, 4, 5, 6, 7]


@pytest.fixture(scope="module")
def prob(oracle_mod):
    return small_problem(oracle_mod, n=101, shuffle=True, field="loguniform")


@pytest.mark.parametrize("bps", [1, 2])
@pytest.mark.parametrize("slv", METHODS)
def test_solve_methods_both_residencies(oracle_mod, prob, bps, slv):
    p = prob
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    mesh.set_blocks_per_sm(bps)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    G, T = mesh.launch_info()
    assert G > 1
    cfg = bief.SlvCfg(slv=slv, nitmax=3000, precon=2, krylov=20 if slv == 7 else 0, eps=1e-10,
                      zero=0.0)
    x = np.zeros(n)
    st, nit, relres = bief.solve(x, A, p["b"].copy(), cfg)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], slv=slv,
                         krylov=20 if slv == 7 else 3, eps=1e-10, nitmax=3000,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == r["status"] and nit == r["nit"] and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    mesh.close()


@pytest.mark.parametrize("bps", [1, 2])
def test_mixed_both_residencies(oracle_mod, prob, bps):
    p = prob
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    mesh.set_blocks_per_sm(bps)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    G, T = mesh.launch_info()
    x = np.zeros(n)
    st, outer, inner, relres = bief.solve_mixed(x, A, p["b"], precon=2, inner_tol=1e-2,
                                                outer_tol=1e-10)
    r = oracle_mod.solve_mixed(p["ik"], p["dm"], "Q", p["xm"], p["b"], precon=2, inner_tol=1e-2,
                               outer_tol=1e-10, max_outer=1000, max_inner=1000000, nblocks=G,
                               nthreads=T)
    assert st == r["status"] == 0 and (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    mesh.close()


@pytest.mark.parametrize("bps", [1, 2])
def test_segment_storage_both_residencies(oracle_mod, prob, bps):
    """Segment storage (STOSEG numbering, the EBE matrix converted by ASSEX3
    on the device): CG and the mixed solve in each residency."""
    p = prob
    n = p["x"].size
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    mesh = bief.Mesh(p["ik"], n)
    mesh.set_blocks_per_sm(bps)
    mesh.set_segments(g1, g2)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    A.to_segments()
    G, T = mesh.launch_info()
    x = np.zeros(n)
    cfg = bief.SlvCfg(slv=1, nitmax=3000, precon=2, krylov=0, eps=1e-10, zero=0.0)
    st, nit, relres = bief.solve(x, A, p["b"].copy(), cfg)
    r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", p["b"], eps=1e-10, nitmax=3000,
                             dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == r["status"] == 0 and nit == r["nit"] and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    x = np.zeros(n)
    st, outer, inner, relres = bief.solve_mixed(x, A, p["b"], precon=2, inner_tol=1e-2,
                                                outer_tol=1e-10)
    r = oracle_mod.solve_mixed_seg(g1, g2, p["dm"], "Q", xa, p["b"], precon=2, inner_tol=1e-2,
                                   outer_tol=1e-10, nblocks=G, nthreads=T)
    assert st == r["status"] == 0 and (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    mesh.close()


def test_residency_argument_checks():
    from opentelemac_b200 import meshgen as mg
    x, y, ik = mg.square_mesh(11)
    mesh = bief.Mesh(ik, x.size)
    for bad in (-1, 3):
        with pytest.raises(bief.BiefError):
            mesh.set_blocks_per_sm(bad)
    mesh.set_blocks_per_sm(0)
    mesh.close()
