"""Segment storage (STO=3) on the device, through the C ABI, against the
oracle: MVSEG for every operation, storage and diagonal type, ASSEX3, the
OMSEG scaling and the whole GRACJG and mixed-precision solves, bit for bit
(the solves with the oracle summing dot products in the device's order)."""
import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu
OPS = ["X=AY    ", "X=X+AY  ", "X=-AY   ", "X=X-AY  ", "X=X+CAY ", "X=CAY   ",
       "X=TAY   ", "X=-TAY  ", "X=X+TAY ", "X=X-TAY ", "X=X+CTAY"]


def _seg_mesh(ik, n):
    g1, g2, es, ori = mg.segments(ik, n)
    mesh = bief.Mesh(ik, n).set_segments(g1, g2)
    return mesh, g1, g2, es, ori


@pytest.mark.parametrize("typext", ["S", "Q", "0"])
@pytest.mark.parametrize("typdia", ["Q", "I", "0"])
def test_mvseg_bitexact(oracle_mod, typdia, typext):
    rng = np.random.default_rng(17)
    x, y, ik = mg.square_mesh(31)
    x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=4)
    n = x.size
    mesh, g1, g2, _, _ = _seg_mesh(ik, n)
    dm = rng.uniform(1, 2, n)
    xa = rng.uniform(-1, 1, (1 if typext != "Q" else 2) * g1.size)
    A = bief.Matrix(mesh).set_seg(dm, xa, typdia, typext)
    assert A.storage == 3
    v, x0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    for op in OPS:
        got = x0.copy()
        bief.matvec(op, got, A, v, c=0.7)
        ref = oracle_mod.mvseg(op, g1, g2, dm, typdia, xa, typext, v, c=0.7, x=x0)
        np.testing.assert_array_equal(got, ref, err_msg=op)


@pytest.mark.parametrize("typext", ["S", "Q"])
def test_assex3_bitexact(oracle_mod, typext):
    rng = np.random.default_rng(5)
    x, y, ik = mg.square_mesh(25)
    x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=8)
    n = x.size
    mesh, g1, g2, es, ori = _seg_mesh(ik, n)
    dm = rng.uniform(1, 2, n)
    xm = rng.uniform(-1, 1, (3 if typext == "S" else 6, ik.shape[0]))
    A = bief.Matrix(mesh, dm, xm, "Q", typext)
    assert A.storage == 1
    A.to_segments()
    assert A.storage == 3
    dm2, xa, td = A.get()
    np.testing.assert_array_equal(dm2, dm)
    ref = oracle_mod.assex3(es, ori, typext, xm, g1.size)
    np.testing.assert_array_equal(xa.ravel(), np.asarray(ref).ravel())


@pytest.mark.parametrize("shuffle,field", [(False, "smooth"), (True, "loguniform")])
def test_solve_seg_bitexact(oracle_mod, shuffle, field):
    p = small_problem(oracle_mod, n=41, shuffle=shuffle, field=field)
    n = p["x"].size
    mesh, g1, g2, es, ori = _seg_mesh(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    b = oracle_mod.mvseg("X=AY    ", g1, g2, p["dm"], "Q", xa, "S", p["xt"])
    A = bief.Matrix(mesh).set_seg(p["dm"], xa, "Q", "S")
    G, T = mesh.launch_info()
    x = np.zeros(n)
    bb = b.copy()
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
    st, nit, relres = bief.solve(x, A, bb, cfg, mutate=True)
    r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", b, eps=1e-10,
                             dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == 0 == r["status"] and nit == r["nit"] and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    # the reference's side effects: B = D.B, A = D.A.D with TYPDIA 'I'
    np.testing.assert_array_equal(bb, r["b"])
    dm2, xa2, td = A.get()
    assert td == "I"
    np.testing.assert_array_equal(xa2.ravel(), r["xa"])


def test_solve_seg_matches_ebe_solve(oracle_mod):
    """The same operator in the two storages: iteration counts within a few
    and solutions within rounding of each other."""
    p = small_problem(oracle_mod, n=61)
    n = p["x"].size
    mesh, g1, g2, es, ori = _seg_mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    cfg = lambda: bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-12, zero=0.0)
    xe = np.zeros(n)
    c1 = cfg()
    bief.solve(xe, A, p["b"], c1)
    A.to_segments()
    xs = np.zeros(n)
    c2 = cfg()
    bief.solve(xs, A, p["b"], c2)
    assert abs(c1.nit - c2.nit) <= 3
    assert np.linalg.norm(xe - xs) / np.linalg.norm(xe) < 1e-10


@pytest.mark.parametrize("field,tol,itol", [("smooth", 1e-8, 0.1), ("loguniform", 1e-10, 1e-4)])
def test_mixed_seg_bitexact(oracle_mod, field, tol, itol):
    p = small_problem(oracle_mod, n=61, field=field)
    n = p["x"].size
    mesh, g1, g2, es, ori = _seg_mesh(p["ik"], n)
    xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    A = bief.Matrix(mesh).set_seg(p["dm"], xa, "Q", "S")
    x = np.zeros(n)
    st, outer, inner, relres = bief.solve_mixed(x, A, p["b"], precon=2, inner_tol=itol,
                                                outer_tol=tol)
    G, T = mesh.launch_info()
    r = oracle_mod.solve_mixed_seg(g1, g2, p["dm"], "Q", xa, p["b"], precon=2, inner_tol=itol,
                                   outer_tol=tol, nblocks=G, nthreads=T)
    assert st == 0 == r["status"]
    assert (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"] <= tol
    np.testing.assert_array_equal(x, r["x"])


def test_segments_reject_bad_numbering():
    x, y, ik = mg.square_mesh(6)
    n = x.size
    g1, g2, _, _ = mg.segments(ik, n)
    mesh = bief.Mesh(ik, n)
    with pytest.raises(bief.BiefError):        # an edge missing
        mesh.set_segments(g1[:-1], g2[:-1])
    with pytest.raises(bief.BiefError):        # an edge twice
        mesh.set_segments(np.r_[g1, g1[:1]], np.r_[g2, g2[:1]])
    bad = g2.copy()
    bad[3] = g1[3]
    with pytest.raises(bief.BiefError):        # a segment of one point
        mesh.set_segments(g1, bad)
    A = bief.Matrix(mesh)
    with pytest.raises(bief.BiefError):        # segment matrix without numbering
        A.set_seg(np.ones(n), np.ones(g1.size))
