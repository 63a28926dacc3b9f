"""bief_solve_noalloc, the SOLVE entry point for callers that cannot
allocate device memory -- for example a Fortran model whose device arrays
belong to an OpenACC/OpenMP data region or to a pool allocator, or a code
that must not call cudaMalloc/cudaFree (with their implicit device
synchronisation) inside its time loop.  It takes the caller's device arrays
and a fixed scratch array compiled into the library, and must give exactly
what the handle-based bief_solve_dev gives, call after call.

This file is collected last on purpose: the test runs after every other
test in a normal run, and also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from opentelemac_b200 import _native, bief, meshgen as mg

pytestmark = pytest.mark.gpu


def _problem(n, seed):
    import torch
    x, y, ik = mg.square_mesh(n, seed=seed)
    coef = mg.wave_coef(mg.depth_loguniform(ik, seed=seed) if seed % 2 else
                        mg.depth_smooth(x, y, ik))
    mesh = bief.Mesh(ik, x.size)
    A = bief.Matrix(mesh)
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    A.assemble_wave(t(x), t(y), t(coef))
    dm, xm, _ = A.get()
    b = np.random.default_rng(seed).uniform(-1, 1, x.size)
    return ik, mesh, A, dm, xm, b


def _cfg(eps=1e-10):
    return bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=eps, zero=0.0)


def _noalloc(ik, dm, xm, b, cfg, nelmax=None, typdia="Q", typext="S"):
    """nelmax > NELEM pads IKLE with node 0 (out of range) and XM with NaN."""
    import torch
    n, ne = dm.size, ik.shape[0]
    nd = 6 if typext == "Q" else 3
    nelmax = ne if nelmax is None else nelmax
    fort = mg.ikle_fortran(ik, nelmax=nelmax).reshape(3, nelmax)
    fort[:, ne:] = 0
    xm_pad = np.full((nd, nelmax), np.nan)
    xm_pad[:, :ne] = np.asarray(xm).reshape(nd, ne)
    d_ikle = torch.tensor(fort.ravel(), device="cuda")
    d_dm = torch.tensor(dm, device="cuda")
    d_xm = torch.tensor(xm_pad, device="cuda")
    d_x = torch.zeros(n, dtype=torch.float64, device="cuda")
    d_b = torch.tensor(b, device="cuda")
    relres = ctypes.c_double()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = _native.lib().bief_solve_noalloc(
        n, ne, nelmax, ctypes.c_void_p(d_ikle.data_ptr()), ctypes.c_void_p(d_dm.data_ptr()),
        ctypes.c_void_p(d_xm.data_ptr()), typdia.encode(), typext.encode(),
        ctypes.c_void_p(d_x.data_ptr()), ctypes.c_void_p(d_b.data_ptr()), ctypes.byref(cfg),
        ctypes.byref(relres), 0, stream)
    torch.cuda.synchronize()
    return st, d_x.cpu().numpy(), d_b.cpu().numpy(), d_dm.cpu().numpy(), d_xm.cpu().numpy(), \
        relres.value


def test_noalloc_matches_handle_solve_twice():
    # calls in a row: a larger mesh after a smaller one, then a smaller one
    # after the larger (whatever the previous call left in the scratch must
    # not reach the next)
    for n, seed in ((101, 4), (181, 7), (61, 8)):
        ik, mesh, A, dm, xm, b = _problem(n, seed)
        ref_cfg = _cfg()
        x_ref, b_ref = np.zeros(dm.size), b.copy()
        st_ref, nit_ref, rel_ref = bief.solve(x_ref, A, b_ref, ref_cfg, mutate=True)
        dm_ref, xm_ref, td = A.get()
        cfg = _cfg()
        st, x, b_out, dm_out, xm_out, rel = _noalloc(ik, dm, xm, b, cfg)
        assert st == st_ref == 0 and cfg.ok == 1
        assert cfg.nit == nit_ref and rel == rel_ref
        np.testing.assert_array_equal(x, x_ref)
        # the reference SOLVE's side effects: B = D.B, A = D.A.D
        np.testing.assert_array_equal(b_out, b_ref)
        np.testing.assert_array_equal(dm_out, dm_ref)
        np.testing.assert_array_equal(xm_out, xm_ref)
        mesh.close()


def test_noalloc_nelmax_padding():
    """IKLE(NELMAX,3) and XM(NELMAX,3) with NELMAX > NELEM: the rows past
    NELEM are neither read (node 0 and NaN there) nor written."""
    ik, mesh, A, dm, xm, b = _problem(61, 3)
    ne = ik.shape[0]
    x_ref, b_ref = np.zeros(dm.size), b.copy()
    st_ref, nit_ref, rel_ref = bief.solve(x_ref, A, b_ref, _cfg(), mutate=True)
    dm_ref, xm_ref, _ = A.get()
    cfg = _cfg()
    st, x, b_out, dm_out, xm_out, rel = _noalloc(ik, dm, xm, b, cfg, nelmax=ne + 29)
    assert st == st_ref == 0 and cfg.nit == nit_ref and rel == rel_ref
    np.testing.assert_array_equal(x, x_ref)
    np.testing.assert_array_equal(b_out, b_ref)
    np.testing.assert_array_equal(dm_out, dm_ref)
    xm_out = xm_out.reshape(3, ne + 29)
    np.testing.assert_array_equal(xm_out[:, :ne], xm_ref)
    assert np.isnan(xm_out[:, ne:]).all()
    mesh.close()


def test_noalloc_rejects_oversize_and_bad_mesh():
    import torch
    L = _native.lib()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    cfg = _cfg()
    st = L.bief_solve_noalloc(65537, 10, 10, p, p, p, b"Q", b"S", p, p, ctypes.byref(cfg), None,
                              0, None)
    assert st == _native.BIEF_ERR_SIZE
    st = L.bief_solve_noalloc(100, 131073, 131073, p, p, p, b"Q", b"S", p, p, ctypes.byref(cfg),
                              None, 0, None)
    assert st == _native.BIEF_ERR_SIZE
    _, _, ik = mg.square_mesh(11)
    fort = mg.ikle_fortran(ik)
    fort[5] = 500                                     # node number outside 1..NPOIN
    d_ikle = torch.tensor(fort, device="cuda")
    d = torch.zeros(121, dtype=torch.float64, device="cuda") + 1.0
    dx = torch.zeros(3 * ik.shape[0], dtype=torch.float64, device="cuda")
    st = L.bief_solve_noalloc(121, ik.shape[0], ik.shape[0], ctypes.c_void_p(d_ikle.data_ptr()),
                              ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(dx.data_ptr()), b"Q",
                              b"S", ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                              ctypes.byref(cfg), None, 0, None)
    assert st == _native.BIEF_ERR_BAD_MESH


def _variant(n, seed, typdia, typext):
    """A symmetric positive definite operator in the given storage: for
    TYPDIA 'I' the wave-equation matrix scaled to a unit diagonal (D A D with
    D = DM^-1/2) and DM = 1 (PRECD1 reads DM even then, and after a PRECON 2
    scaling the solve takes the diagonal as the identity, so DM must be the
    true diagonal); for TYPEXT 'Q' a non-symmetric copy whose upper and
    lower terms differ by up to 1% (a skew-symmetric change, so D.AD > 0
    stays true)."""
    ik, mesh, A, dm, xm, b = _problem(n, seed)
    xm = np.asarray(xm).reshape(3, -1)
    rng = np.random.default_rng(seed + 1)
    if typdia == "I":
        d = 1.0 / np.sqrt(dm)
        xm = np.stack([xm[0] * d[ik[:, 0]] * d[ik[:, 1]], xm[1] * d[ik[:, 0]] * d[ik[:, 2]],
                       xm[2] * d[ik[:, 1]] * d[ik[:, 2]]])
        dm = np.ones(dm.size)
    if typext == "Q":
        s = 0.01 * xm * rng.uniform(-1, 1, xm.shape)
        xm = np.concatenate([xm + s, xm - s])
    A.set(dm, xm, typdia, typext)
    return ik, mesh, A, dm, xm, b


@pytest.mark.parametrize("typext", ["S", "Q"])
@pytest.mark.parametrize("typdia", ["Q", "I"])
@pytest.mark.parametrize("precon", [1, 2, 5])
def test_noalloc_variants_match_handle(precon, typdia, typext):
    """Every storage and preconditioning branch of the kernels behind the
    entry point (the non-symmetric kernel with six off-diagonal columns, no
    change of variables for PRECON 1, |DM| for PRECON 5, both diagonal
    kinds): bit for bit what bief_solve_dev gives, at convergence or at
    NITMAX, side effects included, on two meshes called in a row."""
    for n, seed in ((81, 5), (41, 9)):
        ik, mesh, A, dm, xm, b = _variant(n, seed, typdia, typext)
        cfg_ref = bief.SlvCfg(slv=1, nitmax=400, precon=precon, krylov=0, eps=1e-10, zero=0.0)
        x_ref, b_ref = np.zeros(dm.size), b.copy()
        st_ref, nit_ref, rel_ref = bief.solve(x_ref, A, b_ref, cfg_ref, mutate=True)
        dm_ref, xm_ref, _ = A.get()
        cfg = bief.SlvCfg(slv=1, nitmax=400, precon=precon, krylov=0, eps=1e-10, zero=0.0)
        st, x, b_out, dm_out, xm_out, rel = _noalloc(ik, dm, xm, b, cfg, typdia=typdia,
                                                     typext=typext)
        assert st == st_ref and st >= 0
        assert cfg.nit == nit_ref and cfg.ok == cfg_ref.ok and rel == rel_ref
        np.testing.assert_array_equal(x, x_ref)
        np.testing.assert_array_equal(b_out, b_ref)
        np.testing.assert_array_equal(dm_out, dm_ref)
        np.testing.assert_array_equal(xm_out.reshape(xm_ref.shape), xm_ref)
        mesh.close()


def test_noalloc_valid_solve_after_bad_mesh():
    """A call refused for a bad IKLE leaves nothing behind that changes the
    next, valid call."""
    import torch
    L = _native.lib()
    _, _, ik_bad = mg.square_mesh(11)
    fort = mg.ikle_fortran(ik_bad)
    fort[3] = 0
    d_ikle = torch.tensor(fort, device="cuda")
    d = torch.ones(121, dtype=torch.float64, device="cuda")
    dx = torch.zeros(3 * ik_bad.shape[0], dtype=torch.float64, device="cuda")
    cfg = _cfg()
    st = L.bief_solve_noalloc(121, ik_bad.shape[0], ik_bad.shape[0],
                              ctypes.c_void_p(d_ikle.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                              ctypes.c_void_p(dx.data_ptr()), b"Q", b"S",
                              ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                              ctypes.byref(cfg), None, 0, None)
    assert st == _native.BIEF_ERR_BAD_MESH
    ik, mesh, A, dm, xm, b = _problem(51, 6)
    x_ref, b_ref = np.zeros(dm.size), b.copy()
    st_ref, nit_ref, rel_ref = bief.solve(x_ref, A, b_ref, _cfg(), mutate=True)
    cfg = _cfg()
    st, x, b_out, _, _, rel = _noalloc(ik, dm, xm, b, cfg)
    assert st == st_ref == 0 and cfg.nit == nit_ref and rel == rel_ref
    np.testing.assert_array_equal(x, x_ref)
    np.testing.assert_array_equal(b_out, b_ref)
    mesh.close()


@pytest.mark.parametrize("slv,precon,krylov,want", [
    (1, -1, 0, "ARGS"), (1, -6, 0, "ARGS"), (1, 7, 0, "UNSUPPORTED"), (1, 22, 0, "UNSUPPORTED"),
    (8, 2, 0, "UNSUPPORTED"), (0, 2, 0, "UNSUPPORTED"), (7, 2, 0, "ARGS"), (7, 2, 5, "UNSUPPORTED"),
    (3, 2, 0, "UNSUPPORTED")])
def test_noalloc_config_errors_match_handle(slv, precon, krylov, want):
    """A configuration the path does not take is refused with the code
    bief_solve gives for it (SLV 2..7 are valid there but not here)."""
    import torch
    ik, mesh, A, dm, xm, b = _problem(21, 2)
    code = getattr(_native, "BIEF_ERR_" + want)
    cfg = bief.SlvCfg(slv=slv, nitmax=10, precon=precon, krylov=krylov, eps=1e-8, zero=0.0)
    st, *_ = _noalloc(ik, dm, xm, b, cfg)
    assert st == code
    if slv not in (2, 3, 4, 5, 6) and not (slv == 7 and krylov > 0):
        with pytest.raises(_native.BiefError) as ei:
            bief.solve(np.zeros(dm.size), A, b.copy(), bief.SlvCfg(
                slv=slv, nitmax=10, precon=precon, krylov=krylov, eps=1e-8, zero=0.0))
        assert ei.value.status == code
    mesh.close()
