"""Degenerate meshes, bit for bit against the oracle: a mesh of one
triangle, and a mesh with a node that belongs to no element (a row with its
diagonal only, as a point of NPOIN that no IKLE entry names) -- MATVEC, the
GRACJG solve and the mixed solve, in EBE and segment storage."""
import numpy as np
import pytest

from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu
OPS = ["X=AY    ", "X=TAY   ", "X=X+AY  ", "X=CAY   ", "X=X-TAY "]


def _check(oracle_mod, x, y, ik, dm, xm, seg):
    n = x.size
    rng = np.random.default_rng(n)
    mesh = bief.Mesh(ik, n)
    A = bief.Matrix(mesh, dm, xm, "Q", "S")
    if seg:
        g1, g2, es, ori = mg.segments(ik, n)
        mesh.set_segments(g1, g2)
        A.to_segments()
        xa = oracle_mod.assex3(es, ori, "S", xm, g1.size)
    yv = rng.uniform(-1, 1, n)
    for op in OPS:
        out0 = rng.uniform(-1, 1, n)
        got = out0.copy()
        bief.matvec(op, got, A, yv, 0.75)
        if seg:
            ref = oracle_mod.mvseg(op, g1, g2, dm, "Q", xa, "S", yv, c=0.75, x=out0)
        else:
            ref = oracle_mod.matvec(op, ik, dm, "Q", xm, "S", yv, c=0.75, x=out0)
        np.testing.assert_array_equal(got, ref, err_msg=op)
    xt = rng.uniform(-1, 1, n)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    G, T = mesh.launch_info()
    sol = np.zeros(n)
    cfg = bief.SlvCfg(slv=1, nitmax=10000, precon=2, krylov=0, eps=1e-12, zero=0.0)
    st, nit, rel = bief.solve(sol, A, b.copy(), cfg)
    kw = dict(eps=1e-12, nitmax=10000, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    r = (oracle_mod.solve_seg(g1, g2, dm, "Q", xa, "S", b, **kw) if seg
         else oracle_mod.solve(ik, dm, "Q", xm, "S", b, **kw))
    assert st == 0 and (st, nit) == (r["status"], r["nit"]) and rel == r["relres"]
    np.testing.assert_array_equal(sol, r["x"])
    np.testing.assert_allclose(sol, xt, rtol=0, atol=1e-8)
    if not seg:
        xm_ = np.zeros(n)
        st, outer, inner, rel = bief.solve_mixed(xm_, A, b, precon=2, inner_tol=0.1,
                                                 outer_tol=1e-10)
        r = oracle_mod.solve_mixed(ik, dm, "Q", xm, b, precon=2, inner_tol=0.1, outer_tol=1e-10,
                                   max_outer=1000, max_inner=1000000, nblocks=G, nthreads=T)
        assert st == 0 == r["status"] and (outer, inner) == (r["outer"], r["inner"])
        np.testing.assert_array_equal(xm_, r["x"])
    mesh.close()


@pytest.mark.parametrize("seg", [False, True])
def test_single_triangle(oracle_mod, seg):
    x = np.array([0.0, 1.0, 0.2])
    y = np.array([0.0, 0.1, 0.9])
    ik = np.array([[0, 1, 2]])
    dm, xm = oracle_mod.wave_matrix(x, y, ik, np.array([5.0 * 9.81]))
    _check(oracle_mod, x, y, ik, dm, xm, seg)


@pytest.mark.parametrize("seg", [False, True])
def test_node_outside_every_element(oracle_mod, seg):
    x, y, ik = mg.square_mesh(11)
    x, y, ik, _, _ = mg.shuffled(x, y, ik)
    dm, xm = oracle_mod.wave_matrix(x, y, ik, mg.wave_coef(mg.depth_smooth(x, y, ik)))
    # one more point, named by no element: its row is its diagonal alone
    x = np.append(x, 2.0)
    y = np.append(y, 2.0)
    dm = np.append(dm, 2.5)
    _check(oracle_mod, x, y, ik, dm, xm, seg)


def test_fan_node_beyond_neighbour_limit(oracle_mod):
    """One node shared by 80 triangles (80 neighbours): the binary64 MATVEC
    and GRACJG (any degree) stay bit-exact; the binary32 operator, which
    holds at most 64 neighbours per node, reports BIEF_ERR_SIZE instead of
    running."""
    import torch
    m = 80
    ang = 2 * np.pi * np.arange(m) / m
    x = np.r_[0.0, np.cos(ang)]
    y = np.r_[0.0, np.sin(ang)]
    ik = np.array([[0, 1 + i, 1 + (i + 1) % m] for i in range(m)])
    dm, xm = oracle_mod.wave_matrix(x, y, ik, np.full(m, 3.0))
    n = x.size
    mesh = bief.Mesh(ik, n)
    A = bief.Matrix(mesh, dm, xm, "Q", "S")
    yv = np.random.default_rng(2).uniform(-1, 1, n)
    got = np.zeros(n)
    bief.matvec("X=AY    ", got, A, yv)
    np.testing.assert_array_equal(got, oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", yv))
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", yv)
    G, T = mesh.launch_info()
    sol = np.zeros(n)
    cfg = bief.SlvCfg(slv=1, nitmax=10000, precon=2, krylov=0, eps=1e-12, zero=0.0)
    st, nit, rel = bief.solve(sol, A, b.copy(), cfg)
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, eps=1e-12, nitmax=10000,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == 0 and (nit, rel) == (r["nit"], r["relres"])
    np.testing.assert_array_equal(sol, r["x"])
    with pytest.raises(bief.BiefError) as e:
        bief.solve_mixed(np.zeros(n), A, b)
    assert e.value.status == -9
    y32 = torch.tensor(yv, dtype=torch.float32, device="cuda")
    with pytest.raises(bief.BiefError) as e:
        bief.matvec32(torch.empty_like(y32), A, y32)
    assert e.value.status == -9
    mesh.close()
