"""Device-path behaviour: the entry points run on the caller's stream
(MATVEC, GRACJG, the mixed solve and the binary32 MATVEC issued on a
non-default stream, inputs produced asynchronously on it just before, give
the default stream's bits); two handles in one process share no state; the
device read-back of the stored matrix equals the host read-back."""
import numpy as np
import pytest

from conftest import small_problem
from opentelemac_b200 import bief

pytestmark = pytest.mark.gpu


def _run(p, stream):
    import torch
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    bh, yh = t(p["b"]), t(p["xt"])
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        # inputs produced on the stream itself, right before the calls
        b = bh * 1.0
        y = yh * 1.0
        out = torch.empty_like(y)
        bief.matvec("X=AY    ", out, A, y)
        x = torch.zeros_like(b)
        cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
        st, nit, rel = bief.solve(x, A, b, cfg)
        xm = torch.zeros_like(b)
        stm, outer, inner, relm = bief.solve_mixed(xm, A, b, precon=2, inner_tol=0.1,
                                                   outer_tol=1e-9)
        y32 = y.float()
        o32 = torch.empty_like(y32)
        bief.matvec32(o32, A, y32)
        res = [v.cpu().numpy() for v in (out, x, xm, o32)]
    stream.synchronize()
    mesh.close()
    return res, (st, nit, rel, stm, outer, inner, relm)


def test_non_default_stream_matches_default(oracle_mod):
    import torch
    p = small_problem(oracle_mod, n=81, shuffle=True, field="loguniform")
    ref, sref = _run(p, torch.cuda.current_stream())
    got, sgot = _run(p, torch.cuda.Stream())
    assert sref == sgot and sref[0] == 0 and sref[3] == 0
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(a, b)


def test_two_handles_share_no_state(oracle_mod):
    """Two meshes in one process, calls interleaved on one stream: solving
    and re-assembling on one handle leaves the other's results unchanged."""
    import torch
    pa = small_problem(oracle_mod, n=41, shuffle=True)
    pb = small_problem(oracle_mod, n=61, field="loguniform")
    ha, hb = bief.Mesh(pa["ik"], pa["x"].size), bief.Mesh(pb["ik"], pb["x"].size)
    A = bief.Matrix(ha, pa["dm"], pa["xm"], "Q", "S")
    B = bief.Matrix(hb, pb["dm"], pb["xm"], "Q", "S")
    cfg = lambda: bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)

    def solve_a():
        x = np.zeros(pa["x"].size)
        st = bief.solve(x, A, pa["b"].copy(), cfg())
        xm = np.zeros(pa["x"].size)
        sm = bief.solve_mixed(xm, A, pa["b"], precon=2, inner_tol=0.1, outer_tol=1e-9)
        return x, xm, st, sm

    first = solve_a()
    xb = np.zeros(pb["x"].size)
    bief.solve(xb, B, pb["b"].copy(), cfg(), mutate=True)          # B's matrix becomes D.B.D
    bief.solve_mixed(np.zeros(pb["x"].size), B, pb["b"], precon=2, inner_tol=1e-4,
                     outer_tol=1e-9)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    B.assemble_wave(t(pb["x"]), t(pb["y"]), t(pb["coef"]))            # and is re-assembled
    again = solve_a()
    for a, b in zip(first[:2], again[:2]):
        np.testing.assert_array_equal(a, b)
    assert first[2:] == again[2:]
    ha.close()
    hb.close()


@pytest.mark.parametrize("seg", [False, True])
def test_device_read_back_equals_host_read_back(oracle_mod, seg):
    """bief_get_matrix_dev returns the bits bief_get_matrix returns, after a
    solve that leaves D.A.D in the handle (SOLVE's side effect), in both
    storages."""
    from opentelemac_b200 import meshgen as mg
    p = small_problem(oracle_mod, n=31, shuffle=True)
    n = p["x"].size
    mesh = bief.Mesh(p["ik"], n)
    A = bief.Matrix(mesh, p["dm"], p["xm"], "Q", "S")
    if seg:
        g1, g2, _, _ = mg.segments(p["ik"], n)
        mesh.set_segments(g1, g2)
        A.to_segments()
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, krylov=0, eps=1e-10, zero=0.0)
    bief.solve(np.zeros(n), A, p["b"].copy(), cfg, mutate=True)
    dm_h, xm_h, td = A.get()
    assert td == "I"
    dm_d, xm_d = A.get_dev()
    np.testing.assert_array_equal(dm_d.cpu().numpy(), dm_h)
    np.testing.assert_array_equal(xm_d.cpu().numpy(), xm_h)
    mesh.close()


def test_segment_matrix_from_device_arrays(oracle_mod):
    """A segment-storage matrix set from device tensors
    (bief_set_matrix_seg_dev) holds and multiplies exactly as the same
    matrix set from host arrays."""
    import torch
    from opentelemac_b200 import meshgen as mg
    p = small_problem(oracle_mod, n=31, shuffle=True)
    n = p["x"].size
    g1, g2, es, ori = mg.segments(p["ik"], n)
    xa = np.ascontiguousarray(oracle_mod.assex3(es, ori, "Q",
                                                np.concatenate([p["xm"], 1.1 * p["xm"]]),
                                                g1.size))
    y = np.random.default_rng(9).uniform(-1, 1, n)
    outs = []
    for dev in (False, True):
        mesh = bief.Mesh(p["ik"], n)
        mesh.set_segments(g1, g2)
        t = (lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")) if dev else (lambda a: a)
        A = bief.Matrix(mesh).set_seg(t(p["dm"]), t(xa), "Q", "Q")
        o = np.zeros(n)
        bief.matvec("X=AY    ", o, A, y)
        dm, xm, _ = A.get()
        outs.append((o, dm, xm))
        mesh.close()
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)
