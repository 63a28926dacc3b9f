"""GMRES (SOLVE with SLV=7, KRYLOV <= 20): the oracle's restatement of
gmres.f against scipy on symmetric and non-symmetric operators in both
storages, and the device kernel bit for bit against the oracle (GPU)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg


def _nonsym(p, seed=2):
    rng = np.random.default_rng(seed)
    xm = p["xm"]
    return np.concatenate([xm, xm * (1 + 0.3 * rng.uniform(-1, 1, xm.shape))])


@pytest.mark.parametrize("typext", ["S", "Q"])
def test_gmres_oracle_vs_scipy(oracle_mod, typext):
    p = small_problem(oracle_mod, n=21, shuffle=True)
    n = p["x"].size
    xm = p["xm"] if typext == "S" else _nonsym(p)
    eye = np.eye(n)
    A = np.stack([oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", xm, typext, eye[:, j])
                  for j in range(n)], axis=1)
    b = A @ p["xt"]
    xs = spla.spsolve(sp.csc_matrix(A), b)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, slv=7, krylov=20, eps=1e-10)
    assert r["status"] == 0 and r["relres"] < 1e-10
    # GMRES minimises the residual: the true scaled residual matches its
    # estimate, and the error is bounded by the condition number (~1e5 here)
    d = 1.0 / np.sqrt(p["dm"])
    true = np.linalg.norm((b - A @ r["x"]) * d) / np.linalg.norm(b * d)
    assert true < 1.05e-10
    assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-4
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    rs = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, slv=7, krylov=20, eps=1e-10)
    assert rs["status"] == 0
    assert np.linalg.norm(rs["x"] - xs) / np.linalg.norm(xs) < 1e-4


def test_gmres_krylov_bounds(oracle_mod):
    p = small_problem(oracle_mod, n=11)
    for k in (0, 21):
        assert oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], slv=7,
                                krylov=k)["status"] == -1


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("typext", ["S", "Q"])
def test_gmres_gpu_bitexact(oracle_mod, storage, typext):
    p = small_problem(oracle_mod, n=41, shuffle=True, field="loguniform")
    n = p["x"].size
    xm = p["xm"] if typext == "S" else _nonsym(p)
    b = oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", xm, typext, p["xt"])
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], xm, "Q", typext)
    if storage == "seg":
        g1, g2, es, ori = mg.segments(p["ik"], n)
        mesh.set_segments(g1, g2)
        A.to_segments()
        xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    G, T = mesh.launch_info()
    for krylov, eps, nitmax in [(20, 1e-8, 10000), (5, 1e-8, 10000), (1, 1e-10, 4),
                                (8, 1e-14, 3)]:
        x = np.zeros(n)
        cfg = bief.SlvCfg(slv=7, nitmax=nitmax, precon=2, krylov=krylov, eps=eps, zero=0.0)
        st, nit, relres = bief.solve(x, A, b.copy(), cfg)
        kw = dict(slv=7, krylov=krylov, eps=eps, nitmax=nitmax,
                  dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
        if storage == "seg":
            r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, **kw)
        else:
            r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, **kw)
        assert (st, nit) == (r["status"], r["nit"]), (krylov, eps)
        assert relres == r["relres"]
        np.testing.assert_array_equal(x, r["x"])
        if eps == 1e-8:
            assert st == 0                              # converged


@pytest.mark.gpu
def test_gmres_krylov_rejected():
    x, y, ik = mg.square_mesh(9)
    mesh = bief.Mesh(ik, x.size)
    A = bief.Matrix(mesh, np.ones(x.size) * 4, np.ones((3, ik.shape[0])) * -0.1, "Q", "S")
    for k in (0, 21):
        with pytest.raises(bief.BiefError) as e:
            bief.solve(np.zeros(x.size), A, np.ones(x.size),
                       bief.SlvCfg(slv=7, nitmax=10, precon=2, krylov=k, eps=1e-8, zero=0.0))
        assert e.value.status == -1
