"""Segment (edge) storage, MATRIX STORAGE = 3: the oracle's restatements of
STOSEG, ASSEX3, MVSEG and SOLVE on segments checked against independent
computations, and the product's segment numbering against the oracle's
STOSEG."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from opentelemac_b200 import meshgen as mg

OPS = ["X=AY    ", "X=X+AY  ", "X=-AY   ", "X=X-AY  ", "X=X+CAY ", "X=CAY   ",
       "X=TAY   ", "X=-TAY  ", "X=X+TAY ", "X=X-TAY ", "X=X+CTAY"]


def _mesh(n, shuffle):
    x, y, ik = mg.square_mesh(n)
    if shuffle:
        x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=5)
    return x, y, ik


@pytest.mark.parametrize("n,shuffle", [(5, False), (21, False), (21, True), (40, True)])
def test_numbering_matches_stoseg(oracle_mod, n, shuffle):
    x, y, ik = _mesh(n, shuffle)
    g1, g2, es, ori = mg.segments(ik, x.size)
    be, bf = mg.boundary_faces(ik)
    o1, o2, oes, oori = oracle_mod.stoseg(ik, x.size, be, bf)
    assert g1.size == 3 * (n - 1) ** 2 + 2 * (n - 1)          # edges of the triangulation
    for a, b in [(g1, o1), (g2, o2), (es, oes), (ori, oori)]:
        np.testing.assert_array_equal(a, b)
    nb = be.size
    assert nb == 4 * (n - 1)
    assert np.all(g1[nb:] < g2[nb:])                          # interior: ordered by node
    # every face is its segment, in the orientation ORISEG says
    a = ik.T.ravel()
    b = ik[:, [1, 2, 0]].T.ravel()
    s = es.ravel()
    first = np.where(ori.ravel() == 1, g1[s], g2[s])
    second = np.where(ori.ravel() == 1, g2[s], g1[s])
    np.testing.assert_array_equal(first, a)
    np.testing.assert_array_equal(second, b)


def _dense_seg(n, g1, g2, dm, typdia, xa, typext):
    A = np.zeros((n, n))
    if typdia == "Q":
        A[np.arange(n), np.arange(n)] = dm
    elif typdia == "I":
        A[np.arange(n), np.arange(n)] = 1.0
    if typext != "0":
        x1 = xa if typext == "S" else xa[0]
        x2 = xa if typext == "S" else xa[1]
        np.add.at(A, (g1, g2), x1)
        np.add.at(A, (g2, g1), x2)
    return A


@pytest.mark.parametrize("typext", ["S", "Q", "0"])
@pytest.mark.parametrize("typdia", ["Q", "I", "0"])
def test_mvseg_vs_dense(oracle_mod, typdia, typext):
    rng = np.random.default_rng(11)
    x, y, ik = _mesh(9, True)
    n = x.size
    g1, g2, _, _ = mg.segments(ik, n)
    dm = rng.uniform(1, 2, n)
    xa = rng.uniform(-1, 1, g1.size) if typext == "S" else rng.uniform(-1, 1, (2, g1.size))
    A = _dense_seg(n, g1, g2, dm, typdia, xa, typext)
    v, x0, c = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), -0.3
    for op in OPS:
        M = A.T if "T" in op[2:] else A
        t = M @ v
        exp = {"AY": t, "X+AY": x0 + t, "-AY": -t, "X-AY": x0 - t, "X+CAY": x0 + c * t,
               "CAY": c * t}[op[2:].strip().replace("T", "")]
        got = oracle_mod.mvseg(op, g1, g2, dm, typdia, xa, typext, v, c=c, x=x0)
        np.testing.assert_allclose(got, exp, rtol=0, atol=1e-13, err_msg=op)


@pytest.mark.parametrize("typext", ["S", "Q"])
def test_assex3_same_operator_as_ebe(oracle_mod, typext):
    """Segment storage built by ASSEX3 is the same assembled matrix as the EBE
    storage it came from (to rounding of the two-term sums)."""
    rng = np.random.default_rng(3)
    x, y, ik = _mesh(17, True)
    n = x.size
    g1, g2, es, ori = mg.segments(ik, n)
    dm = rng.uniform(1, 2, n)
    xm = rng.uniform(-1, 1, (3 if typext == "S" else 6, ik.shape[0]))
    xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    A_seg = _dense_seg(n, g1, g2, dm, "Q", xa, typext)
    eye = np.eye(n)
    A_ebe = np.stack([oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, typext, eye[:, j])
                      for j in range(n)], axis=1)
    np.testing.assert_allclose(A_seg, A_ebe, rtol=0, atol=1e-15)


def test_solve_seg_vs_spsolve(oracle_mod, cfg0_problem):
    p = cfg0_problem
    n = p["x"].size
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    Asp = sp.coo_matrix((np.concatenate([p["dm"], xa, xa]),
                         (np.concatenate([np.arange(n), g1, g2]),
                          np.concatenate([np.arange(n), g2, g1]))), shape=(n, n)).tocsr()
    b = oracle_mod.mvseg("X=AY    ", g1, g2, p["dm"], "Q", xa, "S", p["xt"])
    xs = spla.spsolve(Asp.tocsc(), b)
    r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", b, eps=1e-12)
    assert r["status"] == 0 and r["typdia"] == "I"
    assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-7
    # the EBE and segment solves of the same operator agree to rounding
    e = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", b, eps=1e-12)
    assert abs(e["nit"] - r["nit"]) <= 3
    assert np.linalg.norm(e["x"] - r["x"]) / np.linalg.norm(e["x"]) < 1e-9
    # SOLVE's side effects on segment storage: XA <- D XA D, B <- D B
    d = 1.0 / np.sqrt(p["dm"])
    np.testing.assert_array_equal(r["xa"], xa * d[g1] * d[g2])
    np.testing.assert_array_equal(r["b"], b * d)


def test_mixed_seg_converges(oracle_mod, cfg0_problem):
    p = cfg0_problem
    n = p["x"].size
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    b = oracle_mod.mvseg("X=AY    ", g1, g2, p["dm"], "Q", xa, "S", p["xt"])
    m = oracle_mod.solve_mixed_seg(g1, g2, p["dm"], "Q", xa, b, outer_tol=1e-10)
    f = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", b, eps=1e-10)
    assert m["status"] == 0 and m["relres"] <= 1e-10
    assert m["inner"] <= 1.3 * f["nit"] + 5
    assert np.linalg.norm(m["x"] - f["x"]) / np.linalg.norm(f["x"]) < 1e-6


def test_single_triangle_numbering(oracle_mod):
    """A mesh of one triangle has boundary segments only (no interior edge
    to number): the product's numbering still equals STOSEG's."""
    ik = np.array([[0, 1, 2]])
    g1, g2, es, ori = mg.segments(ik, 3)
    be, bf = mg.boundary_faces(ik)
    o1, o2, oes, oori = oracle_mod.stoseg(ik, 3, be, bf)
    for a, b in [(g1, o1), (g2, o2), (es, oes), (ori, oori)]:
        np.testing.assert_array_equal(a, b)
    assert g1.size == 3
