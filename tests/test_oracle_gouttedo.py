"""The restatement on the reference's own gouttedo mesh (tests/golden/
gouttedo.npz, 4,624 nodes in the reference's numbering): the operator
frozen for the device tests is the one PROPAG builds, and the compensated
GRACJG (FINITE ELEMENT ASSEMBLY 3, as the case runs) gives the same bits in
the reference's sequential dot order and in the device's blocked order."""
import numpy as np

from conftest import GOUTTEDO_DT, GOUTTEDO_TETA, GRAV, gouttedo_problem


def test_gouttedo_operator_is_propags(oracle_mod):
    """Symmetric positive diagonal, diffusion rows summing to zero (A 1 is
    the mass matrix's row sums over DT), the case's TETA and DT in DM1."""
    p = gouttedo_problem(oracle_mod)
    one = np.ones(p["x"].size)
    dmm, xmm = oracle_mod.mass_diff_matrix(p["x"], p["y"], p["ik"], 0.0 * p["dm1"], p["h"],
                                           kind=12, xmul_mass=1.0 / GOUTTEDO_DT, xmul_dif=-1.0)
    a1 = oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", p["xm"], "S", one)
    m1 = oracle_mod.matvec("X=AY    ", p["ik"], dmm, "Q", xmm, "S", one)
    np.testing.assert_allclose(a1, m1, rtol=1e-9, atol=1e-9 * np.abs(p["dm"]).max())
    assert p["dm1"][0] == -GOUTTEDO_TETA * GOUTTEDO_TETA * GRAV * GOUTTEDO_DT
    assert (p["dm"] > 0).all() and (p["h"] >= 2.4).all() and p["h"].max() <= 4.8


def test_gouttedo_compensated_solve_order_independent(oracle_mod):
    p = gouttedo_problem(oracle_mod)
    for precon, eps, nitmax in ((0, 1e-4, 100), (2, 1e-12, 100000)):
        seq = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], precon=precon,
                               eps=eps, nitmax=nitmax, dot_mode=oracle_mod.DOT_COMP_SEQUENTIAL)
        blk = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], precon=precon,
                               eps=eps, nitmax=nitmax, dot_mode=oracle_mod.DOT_COMP_BLOCKED,
                               nblocks=3, nthreads=1024)
        assert seq["status"] == blk["status"] and seq["nit"] == blk["nit"]
        assert seq["relres"] == blk["relres"]
        np.testing.assert_array_equal(seq["x"], blk["x"])
    # the case's own settings converge within its 100 iterations
    assert seq["status"] == 0
