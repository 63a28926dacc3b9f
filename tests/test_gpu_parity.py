"""Device kernels (through the C ABI) against the CPU oracle.

Bit-exact: MATVEC (every operation, storage and diagonal type), the PRECD1
change of variables, the wave-operator assembly, and the whole GRACJG solve
when the oracle sums dot products in the device's block/tree order.
Against the reference's sequential dot order the solve agrees to the
rounding-level tolerance documented in each test."""
import os

import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
OPS = ["X=AY    ", "X=X+AY  ", "X=-AY   ", "X=X-AY  ", "X=X+CAY ", "X=CAY   ",
       "X=TAY   ", "X=-TAY  ", "X=X+TAY ", "X=X-TAY ", "X=X+CTAY"]


def cfg(nitmax=100000, eps=1e-8, precon=2, slv=1):
    return bief.SlvCfg(slv=slv, nitmax=nitmax, precon=precon, krylov=0, eps=eps, zero=0.0)


@pytest.mark.parametrize("typext", ["S", "Q", "0"])
@pytest.mark.parametrize("typdia", ["Q", "I", "0"])
def test_matvec_bitexact(oracle_mod, typdia, typext):
    rng = np.random.default_rng(7)
    x, y, ik = mg.square_mesh(31)
    x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=3)
    n, ne = x.size, ik.shape[0]
    dm = rng.uniform(1, 2, n)
    xm = rng.uniform(-1, 1, (6 if typext == "Q" else 3, ne))
    mesh = bief.Mesh(ik, n)
    A = bief.Matrix(mesh, dm, xm, typdia, typext)
    v = rng.uniform(-1, 1, n)
    x0 = rng.uniform(-1, 1, n)
    for op in OPS:
        got = x0.copy()
        bief.matvec(op, got, A, v, c=-0.3)
        ref = oracle_mod.matvec(op, ik, dm, typdia, xm, typext, v, c=-0.3, x=x0)
        np.testing.assert_array_equal(got, ref, err_msg=op)
    # X aliasing Y is allowed (the reference goes through MESH%T)
    got = v.copy()
    bief.matvec("X=X+AY  ", got, A, got)
    np.testing.assert_array_equal(got, oracle_mod.matvec("X=X+AY  ", ik, dm, typdia, xm,
                                                         typext, v, x=v))


def _fan_mesh(nfan=300):
    """A 41 x 41 grid plus a disc of nfan triangles around one more node
    (numbered after the grid, its ring after it): that centre node is in
    nfan elements."""
    x, y, ik = mg.square_mesh(41)
    n = x.size
    t = 2 * np.pi * np.arange(nfan) / nfan
    xf = np.concatenate([x, [20.5], 20.5 + 3 * np.cos(t)])
    yf = np.concatenate([y, [-5.0], -5.0 + 3 * np.sin(t)])
    ring = n + 1 + np.arange(nfan)
    fan = np.stack([np.full(nfan, n), ring, np.roll(ring, -1)], axis=1)
    return xf, yf, np.concatenate([ik, fan]).astype(np.int32)


def _mesh_for(form):
    if form.startswith("fan"):
        return _fan_mesh(int(form[3:]))
    x, y, ik = mg.square_mesh(201)
    if form == "band":      # row-wise nodes, elements in random order
        ik = ik[np.random.default_rng(5).permutation(ik.shape[0])]
    elif form == "any":     # nodes and elements in random order
        x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=5)
    elif form == "ikle":
        x, y, ik = _fan_mesh()
    return x, y, ik


@pytest.mark.parametrize("form,expect", [("local", "local"), ("band", "band"), ("any", "any"),
                                         ("ikle", "ikle"), ("fan255", "local"),
                                         ("fan256", "ikle")])
def test_matvec_bitexact_every_record_format(oracle_mod, form, expect):
    """MATVEC reads the most compact gather records the numbering allows: a
    201 x 201 mesh in row-wise numbering fits 16-bit element and vertex
    offsets ('local'); with its elements in random order only the vertex
    offsets fit ('band'); renumbered at random, neither ('any'); a node in
    300 triangles leaves the product to read IKLE ('ikle'); the limit is
    255 entries per node (a fan of 255 triangles keeps the 6-byte records,
    256 does not).  Every operation is bit for bit the oracle's in each."""
    rng = np.random.default_rng(8)
    x, y, ik = _mesh_for(form)
    n, ne = x.size, ik.shape[0]
    dm = rng.uniform(1, 2, n)
    for typext in ("S", "Q"):
        xm = rng.uniform(-1, 1, (6 if typext == "Q" else 3, ne))
        mesh = bief.Mesh(ik, n)
        assert mesh.matvec_format() == expect
        A = bief.Matrix(mesh, dm, xm, "Q", typext)
        v = rng.uniform(-1, 1, n)
        x0 = rng.uniform(-1, 1, n)
        for op in OPS:
            got = x0.copy()
            bief.matvec(op, got, A, v, c=1.7)
            ref = oracle_mod.matvec(op, ik, dm, "Q", xm, typext, v, c=1.7, x=x0)
            np.testing.assert_array_equal(got, ref, err_msg=f"{op} {typext}")
        mesh.close()


def test_matvec_config0_device_path(oracle_mod, cfg0_problem):
    import torch
    p = cfg0_problem
    mesh = bief.Mesh(p["ik"], p["x"].size)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    y = torch.tensor(p["xt"], device="cuda")
    out = torch.zeros_like(y)
    bief.matvec("X=AY    ", out, A, y)
    np.testing.assert_array_equal(out.cpu().numpy(), p["b"])


def test_assembly_bitexact(oracle_mod):
    import torch
    for shuffle in (False, True):
        p = small_problem(oracle_mod, n=41, shuffle=shuffle, field="loguniform")
        mesh = bief.Mesh(p["ik"], p["x"].size)
        A = bief.Matrix(mesh)
        t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
        A.assemble_wave(t(p["x"]), t(p["y"]), t(p["coef"]))
        dm, xm, td = A.get()
        assert td == "Q"
        np.testing.assert_array_equal(dm, p["dm"])
        np.testing.assert_array_equal(xm, p["xm"])


def _gpu_solve(p, eps=1e-8, precon=2, nitmax=100000, x0=None, mutate=False):
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    x = np.zeros(n) if x0 is None else x0.copy()
    b = p["b"].copy()
    c = cfg(nitmax=nitmax, eps=eps, precon=precon)
    st, nit, relres = bief.solve(x, A, b, c, mutate=mutate)
    return dict(x=x, b=b, status=st, nit=nit, relres=relres, ok=c.ok, mesh=mesh, A=A)


@pytest.mark.parametrize("case", ["cfg0", "shuffled31", "loguniform41"])
def test_solve_bitexact_blocked_order(oracle_mod, cfg0_problem, case):
    p = {"cfg0": lambda: cfg0_problem,
         "shuffled31": lambda: small_problem(oracle_mod, n=31, shuffle=True),
         "loguniform41": lambda: small_problem(oracle_mod, n=41, field="loguniform")}[case]()
    g = _gpu_solve(p)
    G, T = g["mesh"].launch_info()
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-8,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert g["status"] == 0 and g["ok"] == 1
    assert g["nit"] == r["nit"]
    assert g["relres"] == r["relres"]
    np.testing.assert_array_equal(g["x"], r["x"])


def test_solve_vs_reference_order(oracle_mod, cfg0_problem):
    """Against the reference's sequential dot: same iteration count within
    2 at EPS=1e-8 (solutions differ at the CG rounding-sensitivity level,
    bounded by 1e-7 here), and 1e-10 agreement once both are converged to
    EPS=1e-13."""
    p = cfg0_problem
    g = _gpu_solve(p, eps=1e-8)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-8)
    assert abs(g["nit"] - r["nit"]) <= 2
    assert np.linalg.norm(g["x"] - r["x"]) / np.linalg.norm(r["x"]) < 1e-7
    g = _gpu_solve(p, eps=1e-13)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-13)
    assert np.linalg.norm(g["x"] - r["x"]) / np.linalg.norm(r["x"]) < 1e-10


def test_solve_golden_21(oracle_mod):
    gd = np.load(os.path.join(GOLDEN, "golden_21.npz"))
    p = dict(x=gd["x"], ik=gd["ikle0"], dm=gd["dm"], xm=gd["xm"], b=gd["b"])
    g = _gpu_solve(p)
    assert g["mesh"].launch_info() == (1, 1024)
    np.testing.assert_array_equal(g["x"], gd["x_final_blocked"])
    assert g["nit"] == int(gd["nit_final_blocked"])
    for nit in (1, 10):
        gi = _gpu_solve(p, eps=1e-30, nitmax=nit)
        assert gi["status"] == nit
        np.testing.assert_array_equal(gi["x"], gd[f"x_nit{nit}_blocked"])


def test_mutate_inputs(oracle_mod):
    p = small_problem(oracle_mod, n=21)
    g = _gpu_solve(p, mutate=True)
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-8)
    np.testing.assert_array_equal(g["b"], r["b"])
    dm, xm, td = g["A"].get()
    assert td == "I" == r["typdia"]
    np.testing.assert_array_equal(xm, r["xm"])
    np.testing.assert_array_equal(dm, r["dm"])


def test_edge_cases(oracle_mod):
    p = small_problem(oracle_mod, n=15)
    n = p["x"].size
    G = None

    def both(**kw):
        pp = dict(p)
        pp["b"] = kw.pop("b", p["b"])
        g = _gpu_solve(pp, **kw)
        Gt = g["mesh"].launch_info()
        r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", pp["b"],
                             x0=kw.get("x0"), precon=kw.get("precon", 2),
                             nitmax=kw.get("nitmax", 100000), eps=kw.get("eps", 1e-8),
                             dot_mode=oracle_mod.DOT_BLOCKED, nblocks=Gt[0], nthreads=Gt[1])
        return g, r

    g, r = both(b=np.zeros(n), x0=np.ones(n))          # X = 0, no iteration
    assert g["status"] == 0 and g["nit"] == 0 and not g["x"].any()
    g, r = both(b=p["b"] * 1e-6)                        # absolute accuracy mode
    assert g["status"] == 0 and g["nit"] == r["nit"]
    np.testing.assert_array_equal(g["x"], r["x"])
    g, r = both(nitmax=5, eps=1e-30)                    # NITMAX: status = iterations
    assert g["status"] == 5 and g["ok"] == 0
    np.testing.assert_array_equal(g["x"], r["x"])
    for pc in (0, 1, 5):                                # other diagonal options
        g, r = both(precon=pc, eps=1e-10)
        assert g["status"] == 0 and g["nit"] == r["nit"]
        np.testing.assert_array_equal(g["x"], r["x"])
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    with pytest.raises(bief.BiefError) as e:           # method outside the path
        bief.solve(np.zeros(n), A, p["b"].copy(), cfg(slv=8))
    assert e.value.status == -5
    with pytest.raises(bief.BiefError) as e:           # Crout preconditioning
        bief.solve(np.zeros(n), A, p["b"].copy(), cfg(precon=14))
    assert e.value.status == -5
    bad = p["dm"].copy()
    bad[3] = np.nan                                     # NaN in the matrix
    A2 = bief.Matrix(bief.Mesh(p["ik"], n), bad, p["xm"], "Q", "S")
    with pytest.raises(bief.BiefError) as e:
        bief.solve(np.zeros(n), A2, p["b"].copy(), cfg(precon=1))
    assert e.value.status == -3
    neg = -p["dm"]                                      # negative definite: breakdown
    A3 = bief.Matrix(bief.Mesh(p["ik"], n), neg, -p["xm"], "Q", "S")
    with pytest.raises(bief.BiefError) as e:
        bief.solve(np.zeros(n), A3, p["b"].copy(), cfg(precon=1))
    assert e.value.status == -2


def test_solve_device_path_matches_host(oracle_mod, cfg0_problem):
    import torch
    p = cfg0_problem
    g = _gpu_solve(p)
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, torch.tensor(p["dm"], device="cuda"),
                    torch.tensor(p["xm"], device="cuda"), "Q", "S")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    b = torch.tensor(p["b"], device="cuda")
    st, nit, relres = bief.solve(x, A, b, cfg())
    assert st == 0 and nit == g["nit"]
    np.testing.assert_array_equal(x.cpu().numpy(), g["x"])
    np.testing.assert_array_equal(b.cpu().numpy(), p["b"])   # b untouched without mutate


@pytest.mark.parametrize("field,tol,itol", [("smooth", 1e-8, 1e-4), ("loguniform", 1e-10, 1e-4),
                                            ("smooth", 1e-8, 0.1), ("loguniform", 1e-10, 0.1)])
def test_mixed_bitexact(oracle_mod, field, tol, itol):
    p = small_problem(oracle_mod, n=61, field=field)
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    x = np.zeros(n)
    st, outer, inner, relres = bief.solve_mixed(x, A, p["b"], precon=2, inner_tol=itol,
                                                outer_tol=tol)
    G, T = mesh.launch_info()
    r = oracle_mod.solve_mixed(p["ik"], p["dm"], "Q", p["xm"], p["b"], precon=2,
                               inner_tol=itol, outer_tol=tol, max_outer=1000,
                               max_inner=1000000, nblocks=G, nthreads=T)
    assert st == 0 == r["status"]
    assert (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"] and relres <= tol
    np.testing.assert_array_equal(x, r["x"])


@pytest.mark.parametrize("precon", [0, 1, 5])
def test_mixed_bitexact_precon_and_initial_guess(oracle_mod, precon):
    """PRECON 0/1 (no scaling: the kernel's full-diagonal path) and 5
    (|D|), from a nonzero initial guess, on a shuffled numbering."""
    p = small_problem(oracle_mod, n=41, shuffle=True, field="loguniform")
    n = p["x"].size
    x0 = np.random.default_rng(precon).uniform(-1, 1, n)
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    x = x0.copy()
    st, outer, inner, relres = bief.solve_mixed(x, A, p["b"], precon=precon, inner_tol=0.1,
                                                outer_tol=1e-9)
    G, T = mesh.launch_info()
    r = oracle_mod.solve_mixed(p["ik"], p["dm"], "Q", p["xm"], p["b"], x0=x0, precon=precon,
                               inner_tol=0.1, outer_tol=1e-9, max_outer=1000,
                               max_inner=1000000, nblocks=G, nthreads=T)
    assert st == 0 == r["status"]
    assert (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"] and relres <= 1e-9
    np.testing.assert_array_equal(x, r["x"])
    mesh.close()


def test_large_mesh_properties(oracle_mod):
    """501 x 501 (251,001 nodes): size-independent checks -- linearity of
    MATVEC, the returned residual equals an independent binary64 residual,
    and the solution is close to the manufactured one."""
    import torch
    x, y, ik = mg.square_mesh(501)
    coef = mg.wave_coef(mg.depth_smooth(x, y, ik))
    n = x.size
    mesh = bief.Mesh(ik, n)
    A = bief.Matrix(mesh)
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    A.assemble_wave(t(x), t(y), t(coef))
    rng = np.random.default_rng(1)
    u, v = t(rng.uniform(-1, 1, n)), t(rng.uniform(-1, 1, n))
    au, av, auv = torch.zeros_like(u), torch.zeros_like(u), torch.zeros_like(u)
    bief.matvec("X=AY    ", au, A, u)
    bief.matvec("X=AY    ", av, A, v)
    bief.matvec("X=AY    ", auv, A, 2.0 * u - 3.0 * v)
    assert torch.allclose(auv, 2.0 * au - 3.0 * av, rtol=0, atol=1e-9 * au.abs().max().item())
    xt = t(mg.random_solution(n))
    b = torch.zeros_like(xt)
    bief.matvec("X=AY    ", b, A, xt)
    dm, xm, _ = A.get()
    sol = torch.zeros_like(xt)
    st, nit, relres = bief.solve(sol, A, b.clone(), cfg(eps=1e-10))
    assert st == 0 and relres <= 1e-10
    # independent residual in the scaled norm GRACJG uses
    bn, sn = b.cpu().numpy(), sol.cpu().numpy()
    res = bn - oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", sn)
    d = 1.0 / np.sqrt(dm)
    rel = np.linalg.norm(res * d) / np.linalg.norm(bn * d)
    assert rel <= 1.01e-10 and abs(rel - relres) <= 0.05 * relres + 1e-14
    assert np.linalg.norm(sn - xt.cpu().numpy()) / np.sqrt(n) < 1e-3
