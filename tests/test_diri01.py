"""DIRI01 (Dirichlet values on boundary points): the oracle's restatement
yields a system whose solution takes the prescribed values, and the device
reproduces the oracle bit for bit (right-hand side, F and the masked matrix)
in both storages, with and without a mask."""
import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg

KDIR = 5


def _boundary(ik, seed=1):
    be, bf = mg.boundary_faces(ik)
    nbor0 = ik[be, bf].astype(np.int32)                 # boundary points in boundary order
    rng = np.random.default_rng(seed)
    limdir = np.where(rng.uniform(size=nbor0.size) < 0.5, KDIR, 4).astype(np.int32)
    fbor = rng.uniform(-2, 2, nbor0.size)
    return nbor0, limdir, fbor


def test_diri01_oracle_solution_takes_values(oracle_mod):
    p = small_problem(oracle_mod, n=21, shuffle=True)
    n = p["x"].size
    nbor0, limdir, fbor = _boundary(p["ik"])
    sm0 = p["b"].copy()
    xm, sm, f = oracle_mod.diri01(p["ik"], p["dm"], "Q", p["xm"], "S", nbor0, limdir, KDIR,
                                  fbor, sm0, np.zeros(n))
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", xm, "S", sm, eps=1e-13)
    assert r["status"] == 0
    d = limdir == KDIR
    np.testing.assert_allclose(r["x"][nbor0[d]], fbor[d], rtol=0, atol=1e-10)
    np.testing.assert_array_equal(f[nbor0[d]], fbor[d])
    # rows and columns of the Dirichlet points lost their off-diagonal terms
    e = np.zeros(n)
    e[nbor0[d][0]] = 1.0
    col = oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", xm, "S", e)
    assert np.count_nonzero(col) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("storage,typext,masked", [("ebe", "S", False), ("ebe", "Q", True),
                                                   ("seg", "S", True), ("seg", "Q", False)])
def test_diri01_gpu_bitexact(oracle_mod, storage, typext, masked):
    p = small_problem(oracle_mod, n=31, shuffle=True)
    n = p["x"].size
    rng = np.random.default_rng(7)
    xm = p["xm"] if typext == "S" else np.concatenate([p["xm"], p["xm"] * 1.1])
    nbor0, limdir, fbor = _boundary(p["ik"])
    mask = (rng.uniform(size=n) < 0.9).astype(np.float64) if masked else None
    sm0 = rng.uniform(-1, 1, n)
    f0 = rng.uniform(-1, 1, n)
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], xm, "Q", typext)
    if storage == "seg":
        g1, g2, es, ori = mg.segments(p["ik"], n)
        mesh.set_segments(g1, g2)
        A.to_segments()
        xa = oracle_mod.assex3(es, ori, typext, xm, g1.size)
        rx, rsm, rf = oracle_mod.diri01_seg(g1, g2, p["dm"], "Q", xa, typext, nbor0, limdir, KDIR,
                                            fbor, sm0, f0, mask)
    else:
        rx, rsm, rf = oracle_mod.diri01(p["ik"], p["dm"], "Q", xm, typext, nbor0, limdir, KDIR,
                                        fbor, sm0, f0, mask)
    sm, f = sm0.copy(), f0.copy()
    bief.diri01(A, nbor0 + 1, limdir, KDIR, fbor, sm, f, mask)
    np.testing.assert_array_equal(sm, rsm)
    np.testing.assert_array_equal(f, rf)
    _, got, _ = A.get()
    np.testing.assert_array_equal(got.ravel(), np.asarray(rx).ravel())


@pytest.mark.gpu
def test_diri01_rejects_nbor_out_of_range(oracle_mod):
    """An NBOR entry outside 1..NPOIN is reported as BIEF_ERR_BAD_MESH: by the
    host entry point before anything runs, and by the device entry point,
    whose kernels skip the entry instead of writing through it; the
    handle stays usable."""
    import torch
    p = small_problem(oracle_mod, n=21)
    n = p["x"].size
    nbor0, limdir, fbor = _boundary(p["ik"])
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    for bad in (0, n + 1, -5, 10 * n):
        nb = nbor0 + 1
        nb[len(nb) // 2] = bad
        lim = np.full_like(limdir, KDIR)           # every point Dirichlet: the bad one is used
        sm, f = np.zeros(n), np.zeros(n)
        with pytest.raises(bief.BiefError) as e:
            bief.diri01(A, nb, lim, KDIR, fbor, sm, f)
        assert e.value.status == -4
        smd = torch.zeros(n, dtype=torch.float64, device="cuda")
        fd = torch.zeros_like(smd)
        with pytest.raises(bief.BiefError) as e:
            bief.diri01(A, nb, lim, KDIR, fbor, smd, fd)
        assert e.value.status == -4
    # the handle still works
    A2 = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    x = np.zeros(n)
    cfg = bief.SlvCfg(slv=1, nitmax=10000, precon=2, krylov=0, eps=1e-8, zero=0.0)
    st, nit, rel = bief.solve(x, A2, p["b"].copy(), cfg)
    assert st == 0
    mesh.close()
