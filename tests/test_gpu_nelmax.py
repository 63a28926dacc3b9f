"""Arrays dimensioned NELMAX > NELEM, as BIEF_OBJ arrays often are: IKLE
(NELMAX,3) and XM(NELMAX,NDIAG) with rows NELEM+1..NELMAX unused.  The
reference loops run to NELEM with the leading dimension NELMAX
(mv0303.f:117-130, om1111.f:576-580, assvec.f:88-93), so the padding is
never read or written.  The host entry points must do the same: results
equal to the unpadded mesh's bit for bit, the caller's padding left as it
was.  The padding holds out-of-range node numbers and NaN coefficients, so
reading it would show (the host check of IKLE runs before anything reaches
the device)."""
import ctypes

import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import _native, bief, meshgen as mg

pytestmark = pytest.mark.gpu


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _padded(p, extra):
    ik = p["ik"]
    n, ne = p["b"].size, ik.shape[0]
    nmax = ne + extra
    fort = mg.ikle_fortran(ik, nelmax=nmax).reshape(3, nmax)
    fort[:, ne:] = 0                                   # node 0: outside 1..NPOIN
    xm = np.asarray(p["xm"], dtype=np.float64).reshape(3, ne)
    xm_pad = np.full((3, nmax), np.nan)
    xm_pad[:, :ne] = xm
    mesh = bief.Mesh.from_fortran(fort.ravel(), n, ne, nmax)
    return mesh, xm, xm_pad, nmax


@pytest.mark.parametrize("extra", [1, 37])
def test_matvec_and_solve_with_nelmax_pitch(oracle_mod, extra):
    p = small_problem(oracle_mod, n=23, shuffle=True, field="loguniform", seed=5)
    ik, n, ne = p["ik"], p["b"].size, p["ik"].shape[0]
    mesh, xm, xm_pad, nmax = _padded(p, extra)
    A = bief.Matrix(mesh, p["dm"], xm_pad, "Q", "S")

    y = np.random.default_rng(3).standard_normal(n)
    for op in ("X=AY    ", "X=TAY   "):
        out = np.zeros(n)
        bief.matvec(op, out, A, y)
        np.testing.assert_array_equal(
            out, oracle_mod.matvec(op, ik, p["dm"], "Q", p["xm"], "S", y))

    x, b = np.zeros(n), p["b"].copy()
    c = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-9, zero=0.0)
    st, nit, relres = bief.solve(x, A, b, c, mutate=True)
    G, T = mesh.launch_info()
    r = oracle_mod.solve(ik, p["dm"], "Q", p["xm"], "S", p["b"], eps=1e-9,
                         dot_mode=oracle_mod.DOT_BLOCKED, nblocks=G, nthreads=T)
    assert st == 0 and nit == r["nit"] > 5 and relres == r["relres"]
    np.testing.assert_array_equal(x, r["x"])
    np.testing.assert_array_equal(b, r["b"])

    # the raw read-back writes XM(1:NELEM, :) with the NELMAX pitch only
    dm_o = np.empty(n)
    buf = np.full((3, nmax), 7.25)
    td = ctypes.create_string_buffer(2)
    assert _native.lib().bief_get_matrix(mesh.handle, _ptr(dm_o), _ptr(buf), td) == 0
    assert td.value == b"I"
    assert (buf[:, ne:] == 7.25).all()
    np.testing.assert_array_equal(buf[:, :ne], np.asarray(r["xm"]).reshape(3, ne))
    np.testing.assert_array_equal(dm_o, r["dm"])
    dm2, xm2, td2 = A.get()
    assert xm2.shape == (3, ne) and td2 == "I"
    np.testing.assert_array_equal(xm2, buf[:, :ne])


def test_unpadded_xm_on_a_nelmax_mesh(oracle_mod):
    """Matrix.set accepts (3, NELEM) on a NELMAX mesh and pads it itself;
    anything else is refused before it reaches the library."""
    p = small_problem(oracle_mod, n=17, seed=2)
    n = p["b"].size
    mesh, xm, xm_pad, nmax = _padded(p, 10)
    A = bief.Matrix(mesh, p["dm"], xm, "Q", "S")
    y = np.random.default_rng(1).standard_normal(n)
    out = np.zeros(n)
    bief.matvec("X=AY    ", out, A, y)
    np.testing.assert_array_equal(
        out, oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", p["xm"], "S", y))
    with pytest.raises(ValueError):
        A.set(p["dm"], xm[:, :-1], "Q", "S")
    with pytest.raises(ValueError):
        A.set(p["dm"][:-1], xm, "Q", "S")
