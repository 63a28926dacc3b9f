"""RESCJG (SOLVE with SLV=2, conjugate residual), ERRMIN (SLV=4, minimum
error) and CGSQUA (SLV=5, conjugate gradient squared): the oracle's
restatements of rescjg.f, errmin.f and cgsqua.f against scipy in both
storages, and the device kernels bit for bit against the oracle (GPU),
converged and stopped at NITMAX."""
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


# conjugate residual needs a symmetric operator; minimum error (CG on A A^T)
# and conjugate gradient squared take either
@pytest.mark.parametrize("slv,typext", [(2, "S"), (4, "S"), (4, "Q"), (5, "S"), (5, "Q")])
def test_oracle_vs_scipy(oracle_mod, slv, typext):
    p = small_problem(oracle_mod, n=21, shuffle=True)
    n = p["x"].size
    xm = p["xm"] if typext == "S" else _nonsym(p)
    eye = np.eye(n)
    A = np.stack([oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", xm, typext, eye[:, j])
                  for j in range(n)], axis=1)
    b = A @ p["xt"]
    xs = spla.spsolve(sp.csc_matrix(A), b)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, slv=slv, eps=1e-12)
    assert r["status"] == 0 and r["relres"] <= 1e-12
    assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-6
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    rs = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, slv=slv, eps=1e-12)
    assert rs["status"] == 0
    assert np.linalg.norm(rs["x"] - xs) / np.linalg.norm(xs) < 1e-6
    # exact initial guess: stops before the first iteration
    z = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, x0=xs, slv=slv, eps=1e-8)
    assert z["status"] == 0 and z["nit"] == 0


def test_rescjg_nonsymmetric_hits_nitmax(oracle_mod):
    """On a non-symmetric operator conjugate residual loses its minimisation
    property: the oracle stops at NITMAX with a positive status, like the
    reference."""
    p = small_problem(oracle_mod, n=21, shuffle=True)
    xm = _nonsym(p)
    b = oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", xm, "Q", p["xt"])
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, "Q", b, slv=2, eps=1e-10, nitmax=300)
    assert r["status"] == 300 and r["nit"] == 300


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("slv,typext", [(2, "S"), (2, "Q"), (4, "S"), (4, "Q"), (5, "S"),
                                        (5, "Q")])
def test_gpu_bitexact(oracle_mod, storage, slv, typext):
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
    runs = [(1e-14, 20)]
    if not (slv == 2 and typext == "Q"):
        runs.insert(0, (1e-10, 100000))
    for eps, nitmax in runs:
        x = np.zeros(n)
        cfg = bief.SlvCfg(slv=slv, nitmax=nitmax, precon=2, krylov=0, eps=eps, zero=0.0)
        st, nit, relres = bief.solve(x, A, b.copy(), cfg)
        kw = dict(slv=slv, eps=eps, nitmax=nitmax, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G,
                  nthreads=T)
        if storage == "seg":
            r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, **kw)
        else:
            r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, **kw)
        assert (st, nit) == (r["status"], r["nit"]) and relres == r["relres"]
        np.testing.assert_array_equal(x, r["x"])
        if nitmax == 100000:
            assert st == 0
    assert st == 20
    mesh.close()
