"""Failure detection on the device without a GPU fault: a grid barrier that
another block never reaches gives up after its time limit, records the
timeout and returns; the context stays usable (a solve afterwards works)."""
import time

import numpy as np
import pytest

from opentelemac_b200 import _native, bief, meshgen as mg

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_device_stays_usable():
    L = _native.lib()
    t0 = time.perf_counter()
    st = L.bief_selftest_timeout(0, 200_000_000)       # 0.2 s limit
    dt = time.perf_counter() - t0
    assert st == _native.BIEF_ERR_DEVICE_TIMEOUT
    assert 0.15 < dt < 10.0
    assert L.bief_selftest_timeout(0, 10) == _native.BIEF_ERR_ARGS
    # the device still works
    x, y, ik = mg.square_mesh(21)
    mesh = bief.Mesh(ik, x.size)
    A = bief.Matrix(mesh, np.full(x.size, 4.0), np.full((3, ik.shape[0]), -0.1), "Q", "S")
    b = np.ones(x.size)
    sol = np.zeros(x.size)
    st, nit, relres = bief.solve(sol, A, b, bief.SlvCfg(slv=1, nitmax=1000, precon=2, krylov=0,
                                                        eps=1e-10, zero=0.0))
    assert st == 0 and relres <= 1e-10
