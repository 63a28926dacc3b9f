"""MODASS = 3 (compensated dot products, dot_comp.f, which P_DOTS uses for
every method): the oracle's Dot2 in the reference's sequential order and in
the device's blocked order agree with the exact dot product, the compensated
solves give the same bits in both orders, and the device's compensated
solves (GRACJG and the other six methods) reproduce the reference's
sequential-order solves bit for bit (GPU)."""
from fractions import Fraction

import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg


def test_compensated_dots_are_correctly_rounded(oracle_mod):
    rng = np.random.default_rng(0)
    n = 5000
    x = rng.uniform(-1, 1, n) * 10.0 ** rng.integers(-8, 8, n)
    y = rng.uniform(-1, 1, n)
    exact = float(sum(Fraction(a) * Fraction(b) for a, b in zip(x, y)))
    seq = oracle_mod.dot(x, y, mode=oracle_mod.DOT_COMP_SEQUENTIAL)
    for nb, nt in [(1, 256), (7, 256), (5, 1024)]:
        blk = oracle_mod.dot(x, y, mode=oracle_mod.DOT_COMP_BLOCKED, nblocks=nb, nthreads=nt)
        assert blk == seq == exact
    plain = oracle_mod.dot(x, y)
    assert plain != exact                  # the plain sum loses bits on this data


def _problems(oracle_mod):
    out = [small_problem(oracle_mod, n=61, field="loguniform"),
           small_problem(oracle_mod, n=41, shuffle=True)]
    x, y, ik = mg.delaunay_mesh(2500, seed=5)
    dm, xm = oracle_mod.wave_matrix(x, y, ik, mg.wave_coef(mg.depth_smooth(x, y, ik)))
    xt = mg.random_solution(x.size)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    out.append(dict(x=x, y=y, ik=ik, dm=dm, xm=xm, xt=xt, b=b))
    return out


def test_compensated_solve_order_independent(oracle_mod):
    for p in _problems(oracle_mod):
        G = max(1, (p["x"].size + 2047) // 2048)
        seq = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-10,
                               dot_mode=oracle_mod.DOT_COMP_SEQUENTIAL)
        blk = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-10,
                               dot_mode=oracle_mod.DOT_COMP_BLOCKED, nblocks=G, nthreads=1024)
        assert seq["status"] == blk["status"] == 0 and seq["nit"] == blk["nit"]
        np.testing.assert_array_equal(seq["x"], blk["x"])


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
def test_modass3_gpu_matches_reference_order(oracle_mod, storage):
    for p in _problems(oracle_mod):
        n = p["x"].size
        mesh = bief.Mesh(p["ik"], n)
        A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
        if storage == "seg":
            g1, g2, es, ori = mg.segments(p["ik"], n)
            mesh.set_segments(g1, g2)
            A.to_segments()
            xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
        G, T = mesh.launch_info()
        x = np.zeros(n)
        cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
        st, nit, relres = bief.solve(x, A, p["b"].copy(), cfg, modass=3)
        for mode in (oracle_mod.DOT_COMP_BLOCKED, oracle_mod.DOT_COMP_SEQUENTIAL):
            kw = dict(eps=1e-10, dot_mode=mode, nblocks=G, nthreads=T)
            if storage == "seg":
                r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", p["b"], **kw)
            else:
                r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], **kw)
            assert st == r["status"] == 0 and nit == r["nit"] and relres == r["relres"]
            np.testing.assert_array_equal(x, r["x"])



@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("slv", [2, 3, 4, 5, 6])
def test_modass3_other_methods_gpu(oracle_mod, storage, slv):
    """P_DOTS switches to DOT_COMP for every method under MODASS = 3
    (p_dots.f:148-156): RESCJG, EQUNOR, ERRMIN, CGSQUA and CGSTAB with
    compensated dots, converged and at NITMAX, bit for bit against the
    oracle in the device's order and in the reference's sequential order."""
    for p in _problems(oracle_mod)[1:]:
        n = p["x"].size
        mesh = bief.Mesh(p["ik"], n)
        A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
        if storage == "seg":
            g1, g2, es, ori = mg.segments(p["ik"], n)
            mesh.set_segments(g1, g2)
            A.to_segments()
            xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
        G, T = mesh.launch_info()
        for eps, nitmax in ((1e-10, 100000), (1e-14, 15)):
            x = np.zeros(n)
            cfg = bief.SlvCfg(slv=slv, nitmax=nitmax, precon=2, krylov=0, eps=eps, zero=0.0)
            st, nit, relres = bief.solve(x, A, p["b"].copy(), cfg, modass=3)
            for mode in (oracle_mod.DOT_COMP_BLOCKED, oracle_mod.DOT_COMP_SEQUENTIAL):
                kw = dict(slv=slv, eps=eps, nitmax=nitmax, dot_mode=mode, nblocks=G, nthreads=T)
                if storage == "seg":
                    r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", p["b"], **kw)
                else:
                    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], **kw)
                assert (st, nit) == (r["status"], r["nit"]) and relres == r["relres"]
                np.testing.assert_array_equal(x, r["x"])
            assert st == (0 if nitmax > 15 else 15)
        mesh.close()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("krylov", [1, 5, 20])
def test_modass3_gmres_gpu(oracle_mod, storage, krylov):
    """GMRES with compensated dots (the Gram-Schmidt dots and the last
    column's K+1 dots), bit for bit against the oracle in both orders."""
    p = _problems(oracle_mod)[1]
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    if storage == "seg":
        g1, g2, es, ori = mg.segments(p["ik"], n)
        mesh.set_segments(g1, g2)
        A.to_segments()
        xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    G, T = mesh.launch_info()
    for eps, nitmax in ((1e-8, 3000), (1e-14, 4)):
        x = np.zeros(n)
        cfg = bief.SlvCfg(slv=7, nitmax=nitmax, precon=2, krylov=krylov, eps=eps, zero=0.0)
        st, nit, relres = bief.solve(x, A, p["b"].copy(), cfg, modass=3)
        for mode in (oracle_mod.DOT_COMP_BLOCKED, oracle_mod.DOT_COMP_SEQUENTIAL):
            kw = dict(slv=7, krylov=krylov, eps=eps, nitmax=nitmax, dot_mode=mode, nblocks=G,
                      nthreads=T)
            if storage == "seg":
                r = oracle_mod.solve_seg(g1, g2, p["dm"], "Q", xa, "S", p["b"], **kw)
            else:
                r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], **kw)
            assert (st, nit) == (r["status"], r["nit"]) and relres == r["relres"]
            np.testing.assert_array_equal(x, r["x"])
    mesh.close()
