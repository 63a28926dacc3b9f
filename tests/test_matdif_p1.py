"""MT02AA with node (P1) coefficients: MATDIF with U per node
(mt02aa.f:244-279) and MATDIFUV with U and V per node (mt02aa.f:200-240),
the form PROPAG assembles the wave-equation operator with
(propag.F:1407-1408), added to the mass matrix.  The oracle's restatement
against closed-form properties, the device assembly bit for bit against it
(GPU), and a solve through the assembled operator."""
import numpy as np
import pytest

from opentelemac_b200 import bief, meshgen as mg


def _mesh(n=21, shuffle=True):
    x, y, ik = mg.square_mesh(n)
    if shuffle:
        x, y, ik, _, _ = mg.shuffled(x, y, ik)
    return x, y, ik


def test_constant_coefficients_reduce_to_p0(oracle_mod):
    x, y, ik = _mesh()
    n, ne = x.size, ik.shape[0]
    for c in (0.7, 3.7, 250.0):
        dm0, xm0 = oracle_mod.wave_matrix(x, y, ik, np.full(ne, c))
        dm1, xm1 = oracle_mod.mass_diff_matrix(x, y, ik, np.full(n, c), kind=11)
        # MATDIFUV with V = 1: COEF2 = 12 U, COEF1 = XMUL / (48 S)
        dm2, xm2 = oracle_mod.mass_diff_matrix(x, y, ik, np.full(n, c), np.ones(n), kind=12)
        for dm, xm in ((dm1, xm1), (dm2, xm2)):
            np.testing.assert_allclose(xm, xm0, rtol=1e-13, atol=1e-15 * np.abs(xm0).max())
            np.testing.assert_allclose(dm, dm0, rtol=1e-13)
    # kind 10 with unit multipliers is the P0 assembly, bit for bit
    u = np.random.default_rng(1).uniform(1, 5, ne)
    dm0, xm0 = oracle_mod.wave_matrix(x, y, ik, u)
    dm3, xm3 = oracle_mod.mass_diff_matrix(x, y, ik, u, kind=10)
    assert np.array_equal(dm0, dm3) and np.array_equal(xm0, xm3)


@pytest.mark.parametrize("kind", [11, 12])
def test_diffusion_rows_sum_to_zero(oracle_mod, kind):
    """The diffusion part has zero row sums (its diagonals are minus the
    row's other terms), so A 1 is the mass matrix's row sum, and the
    operator scales linearly with XMUL and U."""
    x, y, ik = _mesh()
    n = x.size
    rng = np.random.default_rng(5)
    u, v = rng.uniform(0.5, 4, n), rng.uniform(0.5, 500, n)
    dmm, xmm = oracle_mod.mass_diff_matrix(x, y, ik, np.zeros(n), np.zeros(n), kind=kind)
    one = np.ones(n)
    mass1 = oracle_mod.matvec("X=AY    ", ik, dmm, "Q", xmm, "S", one)
    dm, xm = oracle_mod.mass_diff_matrix(x, y, ik, u, v, kind=kind, xmul_mass=1.0, xmul_dif=9.81)
    a1 = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", one)
    np.testing.assert_allclose(a1, mass1, rtol=1e-9, atol=1e-9 * np.abs(dm).max())
    dmb, xmb = oracle_mod.mass_diff_matrix(x, y, ik, 2 * u, v, kind=kind, xmul_mass=0.0,
                                           xmul_dif=9.81)
    dmc, xmc = oracle_mod.mass_diff_matrix(x, y, ik, u, v, kind=kind, xmul_mass=0.0,
                                           xmul_dif=2 * 9.81)
    np.testing.assert_allclose(xmb, xmc, rtol=1e-14, atol=1e-14 * np.abs(xmb).max())


def test_propag_sign_convention(oracle_mod):
    """PROPAG calls MATDIFUV with XMUL = -1 and U = DM1 < 0 (DM1 = -TETAU
    TETAH GRAV V2DPAR / AM2%D): the result is positive definite."""
    x, y, ik = _mesh(15)
    n = x.size
    rng = np.random.default_rng(9)
    dm1 = -9.81 * rng.uniform(0.5, 2, n)
    hprop = rng.uniform(1, 50, n)
    dm, xm = oracle_mod.mass_diff_matrix(x, y, ik, dm1, hprop, kind=12, xmul_mass=1.0,
                                         xmul_dif=-1.0)
    eye = np.eye(n)
    A = np.stack([oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", eye[:, j])
                  for j in range(n)], axis=1)
    np.testing.assert_allclose(A, A.T, rtol=0, atol=1e-12 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [10, 11, 12])
def test_gpu_assembly_bitexact(oracle_mod, kind):
    import torch
    x, y, ik = _mesh(41)
    n, ne = x.size, ik.shape[0]
    rng = np.random.default_rng(kind)
    u = rng.uniform(0.5, 4, ne if kind == 10 else n)
    v = rng.uniform(0.5, 500, n) if kind == 12 else None
    xmm, xmd = (1.0, -1.0) if kind == 12 else (0.5, 9.81)
    if kind == 12:
        u = -u
    dm_o, xm_o = oracle_mod.mass_diff_matrix(x, y, ik, u, v, kind=kind, xmul_mass=xmm,
                                             xmul_dif=xmd)
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    mesh = bief.Mesh(ik, n)
    A = bief.Matrix(mesh)
    A.assemble_mass_diff(t(x), t(y), t(u), None if v is None else t(v), kind=kind,
                         xmul_mass=xmm, xmul_dif=xmd)
    dm, xm, td = A.get()
    assert td == "Q"
    assert np.array_equal(dm, dm_o)
    assert np.array_equal(xm, xm_o)
    # the assembled operator through the device CG, bit for bit
    xt = mg.random_solution(n)
    b = oracle_mod.matvec("X=AY    ", ik, dm_o, "Q", xm_o, "S", xt)
    G, T = mesh.launch_info()
    xs = np.zeros(n)
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
    st, nit, rel = bief.solve(xs, A, b.copy(), cfg)
    r = oracle_mod.solve(ik, dm_o, "Q", xm_o, "S", b, eps=1e-10,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == 0 and (st, nit) == (r["status"], r["nit"]) and rel == r["relres"]
    np.testing.assert_array_equal(xs, r["x"])
    mesh.close()


@pytest.mark.gpu
def test_gpu_assembly_rejects_bad_kind(oracle_mod):
    import torch
    x, y, ik = _mesh(5, shuffle=False)
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    mesh = bief.Mesh(ik, x.size)
    A = bief.Matrix(mesh)
    with pytest.raises(bief.BiefError) as e:
        A.assemble_mass_diff(t(x), t(y), t(np.ones(x.size)), kind=13)
    assert e.value.status == -1
    mesh.close()
