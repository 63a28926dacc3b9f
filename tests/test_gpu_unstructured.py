"""Unstructured meshes on the device: a Delaunay mesh written to and read
back from a SERAFIN file, then MATVEC, the GRACJG solve, the mixed solve
and segment storage, each bit-exact against the oracle."""
import numpy as np
import pytest

from opentelemac_b200 import bief, meshgen as mg, serafin

pytestmark = pytest.mark.gpu


def _problem(oracle_mod, tmp_path, npts=6000):
    x, y, ik = mg.delaunay_mesh(npts, seed=31)
    p = tmp_path / "geo.slf"
    serafin.mesh_file(p, x, y, ik)
    s = serafin.read(p)
    ik = s.ikle.astype(np.int32)
    coef = mg.wave_coef(mg.depth_loguniform(ik))
    dm, xm = oracle_mod.wave_matrix(s.x, s.y, ik, coef)
    xt = mg.random_solution(s.npoin)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    return s, ik, dm, xm, b


def test_unstructured_ebe_and_mixed(oracle_mod, tmp_path):
    s, ik, dm, xm, b = _problem(oracle_mod, tmp_path)
    mesh = bief.Mesh.from_fortran(s.ikle_fortran(), s.npoin, s.nelem, s.nelem)
    A = bief.Matrix(mesh, dm, xm, "Q", "S")
    v = np.random.default_rng(3).uniform(-1, 1, s.npoin)
    out = np.zeros(s.npoin)
    bief.matvec("X=AY    ", out, A, v)
    np.testing.assert_array_equal(out, oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", v))
    G, T = mesh.launch_info()
    x = np.zeros(s.npoin)
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
    st, nit, relres = bief.solve(x, A, b, cfg)
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, eps=1e-10, dot_mode=oracle_mod.DOT_BLOCKED,
                         nblocks=G, nthreads=T)
    assert st == 0 == r["status"] and nit == r["nit"]
    np.testing.assert_array_equal(x, r["x"])
    xmx = np.zeros(s.npoin)
    st, outer, inner, rel = bief.solve_mixed(xmx, A, b, outer_tol=1e-10)
    m = oracle_mod.solve_mixed(ik, dm, "Q", xm, b, outer_tol=1e-10, max_outer=1000,
                               max_inner=1000000, nblocks=G, nthreads=T)
    assert st == 0 == m["status"] and (outer, inner) == (m["outer"], m["inner"])
    np.testing.assert_array_equal(xmx, m["x"])
    # the solution written as a result file and read back
    res = serafin.Serafin(title="solution", var_names=["X"], var_units=["M"], ikle=s.ikle,
                          x=s.x, y=s.y, times=[0.0], values=[x[None, :]], double=True)
    serafin.write(tmp_path / "res.slf", res)
    back = serafin.read(tmp_path / "res.slf")
    np.testing.assert_array_equal(back.values[0][0], x)


def test_unstructured_segments(oracle_mod, tmp_path):
    s, ik, dm, xm, b = _problem(oracle_mod, tmp_path, npts=4000)
    g1, g2, es, ori = mg.segments(ik, s.npoin)
    mesh = bief.Mesh(ik, s.npoin).set_segments(g1, g2)
    A = bief.Matrix(mesh, dm, xm, "Q", "S").to_segments()
    _, xa, _ = A.get()
    np.testing.assert_array_equal(xa.ravel(), oracle_mod.assex3(es, ori, "S", xm, g1.size))
    G, T = mesh.launch_info()
    x = np.zeros(s.npoin)
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
    st, nit, relres = bief.solve(x, A, b, cfg)
    r = oracle_mod.solve_seg(g1, g2, dm, "Q", xa.ravel(), "S", b, eps=1e-10,
                             dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == 0 == r["status"] and nit == r["nit"]
    np.testing.assert_array_equal(x, r["x"])
