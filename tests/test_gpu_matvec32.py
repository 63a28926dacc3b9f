"""MATVEC 'X=AY' in binary32 (the mixed-precision inner operator applied to
the stored matrix) against a plain PyTorch fp32 product of the same
operator, on EBE and segment storage, TYPDIA 'Q' and 'I'; the lazily built
binary32 copy follows matrix changes and mixed solves."""
import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu


def _dense(oracle_mod, p, dm, typdia):
    n = p["x"].size
    eye = np.eye(n)
    return np.stack([oracle_mod.matvec("X=AY    ", p["ik"], dm, typdia, p["xm"], "S", eye[:, j])
                     for j in range(n)], axis=1)


def _check(x32, A, y):
    """|x - fl32(A) fl32(y)| <= 32 u32 (|A| |y|) row by row, u32 = 2**-24
    (each row sums at most 7 terms, rounded in a different order)."""
    import torch
    A32 = torch.tensor(A, dtype=torch.float32)
    y32 = torch.tensor(y, dtype=torch.float32)
    ref = (A32 @ y32).numpy().astype(np.float64)
    scale = np.abs(A) @ np.abs(y)
    err = np.abs(x32.cpu().numpy().astype(np.float64) - ref)
    assert np.all(err <= 32 * 2.0 ** -24 * scale + 1e-30), float((err / scale).max())


@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("typdia", ["Q", "I"])
def test_matvec32_vs_torch_fp32(oracle_mod, storage, typdia):
    import torch
    p = small_problem(oracle_mod, n=41, shuffle=True, field="loguniform")
    n = p["x"].size
    A = _dense(oracle_mod, p, p["dm"], typdia)
    mesh = bief.Mesh(p["ik"], n)
    M = bief.Matrix(mesh, p["dm"], p["xm"], typdia, "S")
    if storage == "seg":
        g1, g2, _, _ = mg.segments(p["ik"], n)
        mesh.set_segments(g1, g2)
        M.to_segments()
    rng = np.random.default_rng(7)
    y = rng.uniform(-1, 1, n)
    yd = torch.tensor(y, dtype=torch.float32, device="cuda")
    x = torch.empty_like(yd)
    bief.matvec32(x, M, yd)
    _check(x, A, y)
    first = x.clone()
    bief.matvec32(x, M, yd)                          # the copy is reused
    assert torch.equal(x, first)
    # a mixed solve overwrites the binary32 buffers with its scaled
    # operator: the next product rebuilds the stored matrix's copy
    sol = torch.zeros(n, dtype=torch.float64, device="cuda")
    b = torch.tensor(p["b"], dtype=torch.float64, device="cuda")
    bief.solve_mixed(sol, M, b, precon=2, outer_tol=1e-8)
    bief.matvec32(x, M, yd)
    assert torch.equal(x, first)
    # X may alias Y
    z = yd.clone()
    bief.matvec32(z, M, z)
    assert torch.equal(z, first)
    mesh.close()


def test_matvec32_follows_matrix_changes(oracle_mod):
    import torch
    p = small_problem(oracle_mod, n=21, shuffle=True)
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    M = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    y = np.random.default_rng(3).uniform(-1, 1, n)
    yd = torch.tensor(y, dtype=torch.float32, device="cuda")
    x = torch.empty_like(yd)
    bief.matvec32(x, M, yd)
    _check(x, _dense(oracle_mod, p, p["dm"], "Q"), y)
    # new matrix on the same handle: 2 DM, 2 XM
    p2 = dict(p, dm=2 * p["dm"], xm=2 * p["xm"])
    M2 = bief.Matrix(mesh, p2["dm"], p2["xm"], "Q", "S")
    bief.matvec32(x, M2, yd)
    _check(x, _dense(oracle_mod, p2, p2["dm"], "Q"), y)
    # SOLVE with the reference's side effects replaces A by D A D
    cfg = bief.SlvCfg(slv=1, nitmax=10000, precon=2, krylov=0, eps=1e-8, zero=0.0)
    bief.solve(np.zeros(n), M2, p2["b"].copy() * 2, cfg, mutate=True)
    dms, xms, td = M2.get()
    p3 = dict(p, dm=dms, xm=xms.reshape(p["xm"].shape))
    bief.matvec32(x, M2, yd)
    _check(x, _dense(oracle_mod, p3, dms, td), y)
    # non-symmetric storage is outside this operator
    MQ = bief.Matrix(mesh, p["dm"], np.concatenate([p["xm"], p["xm"]]), "Q", "Q")
    with pytest.raises(bief.BiefError) as e:
        bief.matvec32(x, MQ, yd)
    assert e.value.status == -5
    mesh.close()


def _max_offset(ik):
    """Largest |neighbour - node| over the mesh's edges."""
    e = np.concatenate([ik[:, [0, 1]], ik[:, [1, 2]], ik[:, [2, 0]]])
    return int(np.abs(e[:, 0].astype(np.int64) - e[:, 1]).max())


@pytest.mark.parametrize("storage", ["ebe", "seg"])
@pytest.mark.parametrize("numbering", ["rowwise", "shuffled"])
def test_slot_column_forms(oracle_mod, numbering, storage):
    """The binary32 slots (EBE storage, or segment storage with STOSEG's
    numbering) name their neighbours as 16-bit offsets from the node when
    every offset fits (row-wise numbering) and as 32-bit columns otherwise
    (a random renumbering of 40,401 nodes): in both, the mixed solve equals
    the oracle bit for bit and the binary32 MATVEC stays within 32 binary32
    ulps of |A| |y| of the binary64 product."""
    import torch
    p = small_problem(oracle_mod, n=201, shuffle=numbering == "shuffled", field="loguniform")
    n = p["x"].size
    assert (_max_offset(p["ik"]) > 32767) == (numbering == "shuffled")
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    if storage == "seg":
        g1, g2, es, ori = mg.segments(p["ik"], n)
        mesh.set_segments(g1, g2)
        A.to_segments()
        xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
    G, T = mesh.launch_info()
    x = np.zeros(n)
    st, outer, inner, relres = bief.solve_mixed(x, A, p["b"], precon=2, inner_tol=1e-2,
                                                outer_tol=1e-10)
    kw = dict(precon=2, inner_tol=1e-2, outer_tol=1e-10, max_outer=1000, max_inner=1000000,
              nblocks=G, nthreads=T)
    if storage == "seg":
        r = oracle_mod.solve_mixed_seg(g1, g2, p["dm"], "Q", xa, p["b"], **kw)
    else:
        r = oracle_mod.solve_mixed(p["ik"], p["dm"], "Q", p["xm"], p["b"], **kw)
    assert st == r["status"] == 0 and (outer, inner) == (r["outer"], r["inner"])
    np.testing.assert_array_equal(x, r["x"])
    # the stored matrix again (the solve scaled its working copy only)
    y = np.random.default_rng(3).uniform(-1, 1, n)
    x32 = torch.zeros(n, dtype=torch.float32, device="cuda")
    bief.matvec32(x32, A, torch.tensor(y, dtype=torch.float32, device="cuda"))
    ref = oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], "Q", p["xm"], "S", y)
    scale = oracle_mod.matvec("X=AY    ", p["ik"], np.abs(p["dm"]), "Q", np.abs(p["xm"]), "S",
                              np.abs(y))
    err = np.abs(x32.cpu().numpy().astype(np.float64) - ref)
    assert np.all(err <= 32 * 2.0 ** -24 * scale + 1e-30), float((err / scale).max())
    mesh.close()
