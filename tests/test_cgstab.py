"""CGSTAB (SOLVE with SLV=6, BiCGSTAB): the oracle's restatement of
cgstab.f against scipy on symmetric and non-symmetric operators in both
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
def test_cgstab_oracle_vs_scipy(oracle_mod, typext):
    p = small_problem(oracle_mod, n=21, shuffle=True)
    n = p["x"].size
    xm = p["xm"] if typext == "S" else _nonsym(p)
    eye = np.eye(n)
    A = np.stack([oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", xm, typext, eye[:, j])
                  for j in range(n)], axis=1)
    b = A @ p["xt"]
    xs = spla.spsolve(sp.csc_matrix(A), b)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, slv=6, eps=1e-12)
    assert r["status"] == 0 and r["relres"] <= 1e-12
    assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-6
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    rs = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, slv=6, eps=1e-12)
    assert rs["status"] == 0
    assert np.linalg.norm(rs["x"] - xs) / np.linalg.norm(xs) < 1e-6
    # b = 0: XL is raised to 1 (absolute mode) before the RMIN test
    # (cgstab.f:107-116), so the X = 0 shortcut never fires and the solve
    # iterates X towards 0
    z = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, np.zeros(n), x0=np.ones(n), slv=6,
                         eps=1e-10)
    assert z["status"] == 0 and z["nit"] > 0 and np.abs(z["x"]).max() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("typext", ["S", "Q"])
def test_cgstab_gpu_bitexact(oracle_mod, storage, typext):
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
    for eps, nitmax in [(1e-10, 100000), (1e-14, 20)]:
        x = np.zeros(n)
        cfg = bief.SlvCfg(slv=6, nitmax=nitmax, precon=2, krylov=0, eps=eps, zero=0.0)
        st, nit, relres = bief.solve(x, A, b.copy(), cfg)
        kw = dict(slv=6, eps=eps, nitmax=nitmax, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G,
                  nthreads=T)
        if storage == "seg":
            r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, typext, b, **kw)
        else:
            r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, typext, b, **kw)
        assert (st, nit) == (r["status"], r["nit"]) and relres == r["relres"]
        np.testing.assert_array_equal(x, r["x"])
    assert st == 20
