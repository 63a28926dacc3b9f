"""Device entry points refuse tensors the library cannot check itself
(wrong dtype, size, device or layout) before any kernel sees them, and the
host entry points refuse short arrays; a valid call afterwards still works."""
import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief

pytestmark = pytest.mark.gpu


def test_bad_tensors_refused(oracle_mod):
    import torch
    p = small_problem(oracle_mod, n=15)
    n, ne = p["b"].size, p["ik"].shape[0]
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    cfg = bief.SlvCfg(slv=1, nitmax=1000, precon=2, krylov=0, eps=1e-8, zero=0.0)
    b = t(p["b"])
    bad = [
        (torch.zeros(n, device="cuda", dtype=torch.float32), TypeError),   # dtype
        (torch.zeros(n - 1, device="cuda", dtype=torch.float64), ValueError),  # size
        (torch.zeros(2 * n, device="cuda", dtype=torch.float64)[::2], ValueError),  # strided
        (torch.zeros(n, dtype=torch.float64), ValueError),                 # host tensor
    ]
    for x, err in bad:
        with pytest.raises(err):
            bief.solve(x, A, b, cfg)
        with pytest.raises(err):
            bief.solve_mixed(x, A, b)
        with pytest.raises(err):
            bief.matvec("X=AY    ", x, A, b)
    with pytest.raises(TypeError):
        bief.matvec32(torch.zeros(n, device="cuda"), A, torch.zeros(n, device="cuda",
                                                                    dtype=torch.float64))
    with pytest.raises(ValueError):                                        # short b
        bief.solve(torch.zeros(n, device="cuda", dtype=torch.float64), A, b[:-1], cfg)
    with pytest.raises(ValueError):
        bief.Matrix(mesh, t(p["dm"]), t(p["xm"])[:-1], "Q", "S")
    with pytest.raises(ValueError):
        A.assemble_wave(t(p["x"]), t(p["y"]), t(p["coef"][:-1]))
    with pytest.raises(ValueError):
        A.assemble_mass_diff(t(p["x"]), t(p["y"]), t(np.ones(ne)), kind=11)
    # host arrays
    with pytest.raises(ValueError):
        bief.solve_mixed(np.zeros(n), A, p["b"][:-1])
    with pytest.raises(ValueError):
        bief.matvec("X=AY    ", np.zeros(n), A, p["b"][:-1])
    with pytest.raises(ValueError):
        bief.diri01(A, np.arange(1, 4), np.ones(2, dtype=np.int32), 1, np.zeros(3),
                    np.zeros(n), np.zeros(n))
    # nothing was launched with a bad argument: a valid solve still matches
    x = torch.zeros(n, device="cuda", dtype=torch.float64)
    st, nit, rel = bief.solve(x, A, b.clone(), cfg)
    G, T = mesh.launch_info()
    r = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-8, nitmax=1000,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == 0 and nit == r["nit"]
    np.testing.assert_array_equal(x.cpu().numpy(), r["x"])
