"""The CPU oracle (C restatement of the reference routines) against
independent computations: dense element matrices assembled with numpy, the
MATVEC operations as dense products, scipy's sparse direct solve, and the
committed golden fixtures.  No GPU needed."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from conftest import small_problem
from opentelemac_b200 import meshgen as mg

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def dense_elements(x, y, ik, coef):
    """P1 mass + coef * stiffness element matrices from the textbook
    formulas (independent of the Fortran operation order)."""
    X, Y = x[ik], y[ik]
    bb = Y[:, [1, 2, 0]] - Y[:, [2, 0, 1]]
    cc = X[:, [2, 0, 1]] - X[:, [1, 2, 0]]
    area = 0.5 * ((X[:, 1] - X[:, 0]) * (Y[:, 2] - Y[:, 0]) - (X[:, 2] - X[:, 0]) * (Y[:, 1] - Y[:, 0]))
    K = (bb[:, :, None] * bb[:, None, :] + cc[:, :, None] * cc[:, None, :]) / (4 * area)[:, None, None]
    M = area[:, None, None] / 12.0 * (np.ones((3, 3)) + np.eye(3))
    return M + coef[:, None, None] * K


def assemble(ik, Ae, n):
    rows = np.repeat(ik, 3, axis=1).ravel()
    cols = np.tile(ik, (1, 3)).ravel()
    return sp.csr_matrix((Ae.ravel(), (rows, cols)), shape=(n, n))


def ebe_dense(ik, dm, typdia, xm, typext, n):
    """Dense matrix of EBE storage (om1111.f:43-50 column convention)."""
    A = np.zeros((n, n))
    if typdia == "Q":
        A[np.arange(n), np.arange(n)] += dm
    elif typdia == "I":
        A[np.arange(n), np.arange(n)] += 1.0
    if typext in ("S", "Q"):
        pairs = [(0, 1, 0), (0, 2, 1), (1, 2, 2)]
        for k, l, c in pairs:
            np.add.at(A, (ik[:, k], ik[:, l]), xm[c])
            ct = c if typext == "S" else c + 3
            np.add.at(A, (ik[:, l], ik[:, k]), xm[ct])
    return A


def test_wave_matrix_vs_dense(oracle_mod):
    p = small_problem(oracle_mod, n=31, shuffle=True)
    Ae = dense_elements(p["x"], p["y"], p["ik"], p["coef"])
    A = assemble(p["ik"], Ae, p["x"].size).toarray()
    np.testing.assert_allclose(p["dm"], np.diag(A), rtol=1e-13)
    np.testing.assert_allclose(p["xm"][0], Ae[:, 0, 1], rtol=1e-9, atol=1e-14 * np.abs(Ae).max())
    np.testing.assert_allclose(p["xm"][1], Ae[:, 0, 2], rtol=1e-9, atol=1e-14 * np.abs(Ae).max())
    np.testing.assert_allclose(p["xm"][2], Ae[:, 1, 2], rtol=1e-9, atol=1e-14 * np.abs(Ae).max())


OPS = ["X=AY    ", "X=X+AY  ", "X=-AY   ", "X=X-AY  ", "X=X+CAY ", "X=CAY   ",
       "X=TAY   ", "X=-TAY  ", "X=X+TAY ", "X=X-TAY ", "X=X+CTAY"]


@pytest.mark.parametrize("typext", ["S", "Q", "0"])
@pytest.mark.parametrize("typdia", ["Q", "I", "0"])
def test_matvec_ops_vs_dense(oracle_mod, rng, typext, typdia):
    x, y, ik = mg.square_mesh(9)
    x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=5)
    n, ne = x.size, ik.shape[0]
    dm = rng.uniform(1, 2, n)
    xm = rng.uniform(-1, 1, (6 if typext == "Q" else 3, ne))
    A = ebe_dense(ik, dm, typdia, xm, typext, n)
    v = rng.uniform(-1, 1, n)
    x0 = rng.uniform(-1, 1, n)
    c = 0.75
    for op in OPS:
        got = oracle_mod.matvec(op, ik, dm, typdia, xm, typext, v, c=c, x=x0)
        M = A.T if "TAY" in op else A
        t = M @ v
        ref = {"AY": t, "X+AY": x0 + t, "-AY": -t, "X-AY": x0 - t, "X+CAY": x0 + c * t,
               "CAY": c * t}[op.strip()[2:].replace("T", "")]
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12, err_msg=op)


def test_solve_vs_scipy(oracle_mod, cfg0_problem):
    p = cfg0_problem
    n = p["x"].size
    Ae = dense_elements(p["x"], p["y"], p["ik"], p["coef"])
    A = assemble(p["ik"], Ae, n)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], precon=2, eps=1e-12)
    assert r["status"] == 0 and r["relres"] <= 1e-12
    xs = spl.spsolve(A.tocsc(), p["b"])
    assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-7
    assert np.linalg.norm(r["x"] - p["xt"]) / np.linalg.norm(p["xt"]) < 1e-7


def test_solve_config0_iterations(oracle_mod, cfg0_problem):
    p = cfg0_problem
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], precon=2, eps=1e-8)
    assert r["status"] == 0 and r["relat"] == 1
    assert r["relres"] <= 1e-8
    assert 300 < r["nit"] < 600


def test_precd1_side_effects(oracle_mod):
    p = small_problem(oracle_mod, n=11)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], precon=2, eps=1e-8)
    d = 1.0 / np.sqrt(p["dm"])
    assert r["typdia"] == "I"
    np.testing.assert_array_equal(r["b"], p["b"] * d)
    ik = p["ik"]
    np.testing.assert_array_equal(r["xm"][0], p["xm"][0] * d[ik[:, 1]] * d[ik[:, 0]])
    np.testing.assert_array_equal(r["xm"][2], p["xm"][2] * d[ik[:, 2]] * d[ik[:, 1]])
    np.testing.assert_array_equal(r["dm"], p["dm"] * d * d)


def test_edge_cases(oracle_mod):
    p = small_problem(oracle_mod, n=11)
    ik, dm, xm, b = p["ik"], p["dm"], p["xm"], p["b"]
    n = b.size
    # ||B|| < 1e-15: X = 0, no iteration (gracjg.F:194-202)
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", np.zeros(n), x0=np.ones(n))
    assert r["status"] == 0 and r["nit"] == 0 and not r["x"].any()
    # ||B||^2 < 1: absolute accuracy (gracjg.F:204-209)
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b * 1e-6, eps=1e-8)
    assert r["status"] == 0 and r["relat"] == 0
    # NITMAX reached: positive status = iterations
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, nitmax=3, eps=1e-30)
    assert r["status"] == 3 and r["nit"] == 3
    # exact initial guess: converged before the first iteration
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, x0=oracle_mod.solve(ik, dm, "Q", xm, "S", b,
                                                                    eps=1e-14)["x"], eps=1e-6)
    assert r["status"] == 0 and r["nit"] == 0
    # no preconditioning (PRECON 0 -> 1) and |diag| preconditioning
    for pc in (0, 1, 5):
        r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, precon=pc, eps=1e-10)
        assert r["status"] == 0
        np.testing.assert_allclose(r["x"], p["xt"], rtol=0, atol=1e-6)
    # methods and preconditioners outside this path
    assert oracle_mod.solve(ik, dm, "Q", xm, "S", b, slv=8)["status"] == -5
    assert oracle_mod.solve(ik, dm, "Q", xm, "S", b, precon=14)["status"] == -5


def test_blocked_dots(oracle_mod, rng):
    v = rng.uniform(-1, 1, 100003)
    w = rng.uniform(-1, 1, 100003)
    exact = float(np.dot(v.astype(np.longdouble), w.astype(np.longdouble)))
    for nb, nt in [(1, 256), (7, 256), (444, 256), (592, 512)]:
        d = oracle_mod.dot(v, w, oracle_mod.DOT_BLOCKED, nb, nt)
        assert abs(d - exact) < 1e-11
    ints = np.arange(1, 5001, dtype=np.float64)
    assert oracle_mod.dot(ints, np.ones_like(ints), oracle_mod.DOT_BLOCKED, 13, 256) == 5000 * 5001 / 2


def test_blocked_vs_sequential_solution(oracle_mod, cfg0_problem):
    """The dot order changes the iterates at the rounding level only:
    same iteration count at 1e-8, and at a tight tolerance the two
    solutions agree to 1e-10."""
    p = cfg0_problem
    args = (p["ik"], p["dm"], "Q", p["xm"], "S", p["b"])
    s = oracle_mod.solve(*args, eps=1e-8)
    bl = oracle_mod.solve(*args, eps=1e-8, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=20)
    assert abs(s["nit"] - bl["nit"]) <= 2
    assert np.linalg.norm(s["x"] - bl["x"]) / np.linalg.norm(s["x"]) < 1e-7
    s = oracle_mod.solve(*args, eps=1e-13)
    bl = oracle_mod.solve(*args, eps=1e-13, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=20)
    assert np.linalg.norm(s["x"] - bl["x"]) / np.linalg.norm(s["x"]) < 1e-10


def test_mixed_oracle(oracle_mod, cfg0_problem):
    """Mixed precision reaches the binary64 answer: at outer_tol=1e-12 it
    agrees with a tight binary64 solve to 1e-7; at 1e-8 it needs about the
    binary64 CG's iteration count (the binary32 CG keeps its search
    direction across residual replacements)."""
    p = cfg0_problem
    ref = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-14)
    m = oracle_mod.solve_mixed(p["ik"], p["dm"], "Q", p["xm"], p["b"], inner_tol=1e-4,
                               outer_tol=1e-12, nblocks=20)
    assert m["status"] == 0 and m["relres"] <= 1e-12
    assert np.linalg.norm(m["x"] - ref["x"]) / np.linalg.norm(ref["x"]) < 1e-7
    fp = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-8)
    m8 = oracle_mod.solve_mixed(p["ik"], p["dm"], "Q", p["xm"], p["b"], outer_tol=1e-8,
                                nblocks=20)
    assert m8["status"] == 0 and m8["relres"] <= 1e-8
    assert m8["inner"] <= 1.1 * fp["nit"] + 5


def test_golden_21(oracle_mod):
    g = np.load(os.path.join(GOLDEN, "golden_21.npz"))
    p = small_problem(oracle_mod, n=21)
    for k, v in (("x", p["x"]), ("y", p["y"]), ("ikle0", p["ik"]), ("coef", p["coef"]),
                 ("dm", p["dm"]), ("xm", p["xm"]), ("xt", p["xt"]), ("b", p["b"])):
        np.testing.assert_array_equal(g[k], v, err_msg=k)
    ik, dm, xm, b = p["ik"], p["dm"], p["xm"], p["b"]
    for nit in (1, 10):
        r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, nitmax=nit, eps=1e-30)
        np.testing.assert_array_equal(r["x"], g[f"x_nit{nit}"])
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, eps=1e-8)
    np.testing.assert_array_equal(r["x"], g["x_final"])
    assert r["nit"] == int(g["nit_final"])
    np.testing.assert_array_equal(r["b"], g["b_scaled"])
    np.testing.assert_array_equal(r["xm"], g["xm_scaled"])
    np.testing.assert_array_equal(oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", p["xt"]),
                                  g["mv_XAY"])


def test_golden_101(oracle_mod, cfg0_problem):
    import hashlib
    g = np.load(os.path.join(GOLDEN, "golden_101.npz"))
    p = cfg0_problem

    def digest(*arrays):
        h = hashlib.sha256()
        for a in arrays:
            h.update(np.ascontiguousarray(a).tobytes())
        return h.hexdigest()

    assert digest(p["x"], p["y"], p["ik"]) == str(g["mesh_digest"])
    assert digest(p["dm"], p["xm"]) == str(g["matrix_digest"])
    assert digest(p["b"]) == str(g["b_digest"])
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-8)
    np.testing.assert_array_equal(r["x"], g["x_final"])
    assert r["nit"] == int(g["nit_final"])


def test_batch_dot_order(oracle_mod, rng):
    v = rng.uniform(-1, 1, 70001)
    w = rng.uniform(-1, 1, 70001)
    exact = float(np.dot(v.astype(np.longdouble), w.astype(np.longdouble)))
    for npt in (1, 2, 4):
        assert abs(oracle_mod.dot_batch(v, w, 1024, npt) - exact) < 1e-11
    ints = np.arange(1, 3001, dtype=np.float64)
    assert oracle_mod.dot_batch(ints, np.ones_like(ints), 1024, 1) == 3000 * 3001 / 2
