"""CPU-side checks of the C ABI library: it loads without a GPU, exports
every function include/bief_b200.h declares, and rejects bad meshes before
touching the device."""
import ctypes
import os
import re

import numpy as np
import pytest

from opentelemac_b200 import _native, meshgen as mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "bief_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bief_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header():
    names = header_functions()
    assert len(names) >= 15
    L = ctypes.CDLL(_native.LIB)
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_native.EXPORTS) == names


def test_strerror():
    L = _native.lib()
    assert L.bief_strerror(0) == b"ok"
    assert b"NITMAX" in L.bief_strerror(12)
    for s in range(-9, 0):
        assert L.bief_strerror(s) != b"unknown status"


def test_bad_mesh_rejected_on_host():
    """IKLE entries outside 1..NPOIN are caught before any device call."""
    _, _, ik = mg.square_mesh(5)
    fort = mg.ikle_fortran(ik)
    fort[7] = 0
    h = ctypes.c_void_p()
    L = _native.lib()
    st = L.bief_mesh_create(25, ik.shape[0], ik.shape[0], fort.ctypes.data_as(ctypes.c_void_p),
                            0, ctypes.byref(h))
    assert st == _native.BIEF_ERR_BAD_MESH and not h.value
    fort[7] = 26
    st = L.bief_mesh_create(25, ik.shape[0], ik.shape[0], fort.ctypes.data_as(ctypes.c_void_p),
                            0, ctypes.byref(h))
    assert st == _native.BIEF_ERR_BAD_MESH
    st = L.bief_mesh_create(0, ik.shape[0], ik.shape[0], fort.ctypes.data_as(ctypes.c_void_p),
                            0, ctypes.byref(h))
    assert st == _native.BIEF_ERR_ARGS
    st = L.bief_mesh_create(25, ik.shape[0], ik.shape[0] - 1,
                            fort.ctypes.data_as(ctypes.c_void_p), 0, ctypes.byref(h))
    assert st == _native.BIEF_ERR_ARGS
    st = L.bief_mesh_create(25, 0, 0, fort.ctypes.data_as(ctypes.c_void_p), 0,
                            ctypes.byref(h))                      # no elements
    assert st == _native.BIEF_ERR_ARGS
    # beyond the (e << 2 | k) gather encoding: refused before IKLE is read
    big = (1 << 29) + 1
    st = L.bief_mesh_create(25, big, big, fort.ctypes.data_as(ctypes.c_void_p), 0,
                            ctypes.byref(h))
    assert st == _native.BIEF_ERR_SIZE and not h.value


def test_null_handle_calls():
    L = _native.lib()
    assert L.bief_destroy(None) == _native.BIEF_ERR_ARGS
    assert L.bief_launch_info(None, None, None) == _native.BIEF_ERR_ARGS
    assert L.bief_kernel_launches(None) == -1


def test_meshgen_shapes_and_orientation():
    x, y, ik = mg.square_mesh(11)
    assert x.size == 121 and ik.shape == (200, 3)
    X, Y = x[ik], y[ik]
    area = 0.5 * ((X[:, 1] - X[:, 0]) * (Y[:, 2] - Y[:, 0]) - (X[:, 2] - X[:, 0]) * (Y[:, 1] - Y[:, 0]))
    assert (area > 0).all()
    np.testing.assert_allclose(area.sum(), 1.0, rtol=1e-12)
    xs, ys, iks, perm, eperm = mg.shuffled(x, y, ik)
    X, Y = xs[iks], ys[iks]
    area2 = 0.5 * ((X[:, 1] - X[:, 0]) * (Y[:, 2] - Y[:, 0]) - (X[:, 2] - X[:, 0]) * (Y[:, 1] - Y[:, 0]))
    np.testing.assert_allclose(np.sort(area2), np.sort(area))
    f = mg.ikle_fortran(ik, nelmax=210)
    assert f.size == 630 and f.min() == 0 and f.max() == 121


def test_depth_fields():
    x, y, ik = mg.square_mesh(41)
    h = mg.depth_smooth(x, y, ik)
    assert 1.0 <= h.min() and h.max() <= 9.0
    h2 = mg.depth_loguniform(ik)
    assert 0.5 <= h2.min() and h2.max() <= 500.0
    nb = mg.element_neighbours(ik)
    assert ((nb >= 0).sum(axis=1) >= 1).all()


def test_host_xm_nelmax_layout():
    """Matrix._host_xm gives the XM(NELMAX,NDIAG) block the host entry points
    read: (nd, nelem) input padded with zeros, (nd, nelmax) taken as is,
    anything else refused before the library sees it."""
    from types import SimpleNamespace
    from opentelemac_b200 import bief
    A = bief.Matrix.__new__(bief.Matrix)
    A.mesh = SimpleNamespace(nelem=5, nelmax=8, npoin=6)
    xm = np.arange(15, dtype=np.float64).reshape(3, 5)
    out = A._host_xm(xm, 3)
    assert out.shape == (3, 8) and out.flags.c_contiguous
    np.testing.assert_array_equal(out[:, :5], xm)
    assert not out[:, 5:].any()
    full = np.arange(24.0).reshape(3, 8)
    np.testing.assert_array_equal(A._host_xm(full.ravel(), 3), full)
    with pytest.raises(ValueError):
        A._host_xm(np.zeros(14), 3)


def test_argument_checks_before_the_library():
    """What the library cannot check on a device address is checked in
    Python first: a CPU tensor, a wrong size or dtype never reaches a
    kernel.  (CUDA-tensor cases are in tests/test_gpu_validation.py.)"""
    from types import SimpleNamespace
    import torch
    from opentelemac_b200 import bief
    m = SimpleNamespace(npoin=4, nelem=2, device=0)
    with pytest.raises(ValueError):
        bief._dev(torch.zeros(4, dtype=torch.float64), 4, m, "x")
    with pytest.raises(ValueError):
        bief._host_in(np.zeros(3), 4, "b")
    a = bief._host_in([1, 2, 3, 4], 4, "b")
    assert a.dtype == np.float64 and a.flags.c_contiguous
