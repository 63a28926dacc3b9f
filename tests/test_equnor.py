"""EQUNOR (SOLVE with SLV=3, CG on the normal equations): the oracle's
restatement of equnor.f against scipy on symmetric and non-symmetric
operators, in both storages, and the device kernel bit for bit against the
oracle (GPU tests)."""
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


def _dense(oracle_mod, ik, dm, xm, typext):
    n = dm.size
    eye = np.eye(n)
    return np.stack([oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, typext, eye[:, j])
                     for j in range(n)], axis=1)


@pytest.mark.parametrize("typext", ["S", "Q"])
def test_equnor_oracle_vs_scipy(oracle_mod, typext):
    p = small_problem(oracle_mod, n=21, shuffle=True)
    xm = p["xm"] if typext == "S" else _nonsym(p)
    A = _dense(oracle_mod, p["ik"], p["dm"], xm, typext)
    b = A @ p["xt"]
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, slv=3, eps=1e-12, nitmax=100000)
    assert r["status"] == 0 and r["typdia"] == "I"
    xs = spla.spsolve(sp.csc_matrix(A), b)
    assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-8
    # segment storage: the same solve on the ASSEX3 image of the matrix
    g1, g2, es, ori = mg.segments(p["ik"], p["x"].size)
    xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    rs = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, slv=3, eps=1e-12,
                              nitmax=100000)
    assert rs["status"] == 0
    assert np.linalg.norm(rs["x"] - xs) / np.linalg.norm(xs) < 1e-8


def test_equnor_nitmax(oracle_mod):
    p = small_problem(oracle_mod, n=21)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], slv=3, eps=1e-14,
                         nitmax=7)
    assert r["status"] == 7 and r["nit"] == 7


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("typext", ["S", "Q"])
def test_equnor_gpu_bitexact(oracle_mod, storage, typext):
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
    for eps, nitmax in [(1e-10, 100000), (1e-14, 25)]:
        x = np.zeros(n)
        cfg = bief.SlvCfg(slv=3, nitmax=nitmax, precon=2, krylov=0, eps=eps, zero=0.0)
        st, nit, relres = bief.solve(x, A, b.copy(), cfg)
        kw = dict(slv=3, eps=eps, nitmax=nitmax, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G,
                  nthreads=T)
        if storage == "seg":
            r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, **kw)
        else:
            r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, **kw)
        assert st == r["status"] and nit == r["nit"] and relres == r["relres"]
        np.testing.assert_array_equal(x, r["x"])
    assert st == 25                                   # NITMAX reached on the second case
