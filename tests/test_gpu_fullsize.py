"""Parity at the benchmark's own sizes, bit for bit against the oracle.

- 1001 x 1001 nodes (1,002,001 nodes, 2,000,000 triangles, smooth depth):
  the on-device assembly, MATVEC 'X=AY', the binary64 GRACJG solve to
  relres 1e-8 (1,927 iterations) and the mixed-precision solve (refinement
  threshold 0.1, the headline workload): every bit of the solution, the
  iteration counts and the residual, against the restatement run in the
  device's dot order -- with one block per SM (148 blocks) and with two
  (296 blocks, the kernels built for half the registers).
- The 256-mesh batch (node counts log-uniform in [2,000, 200,000], one
  persistent launch): the smallest, the median and the largest instance
  against the restatement of the batched algorithm in the batched dot order.

The oracle runs these on all host threads (oracle.threads); the threaded
restatement gives the same bits as the sequential one
(tests/test_oracle_threads.py)."""
import numpy as np
import pytest

from opentelemac_b200 import bief, meshgen as mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wave1m(oracle_mod):
    x, y, ik = mg.square_mesh(1001)
    coef = mg.wave_coef(mg.depth_smooth(x, y, ik))
    dm, xm = oracle_mod.wave_matrix(x, y, ik, coef)
    xt = mg.random_solution(x.size)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    return dict(x=x, y=y, ik=ik, coef=coef, dm=dm, xm=xm, xt=xt, b=b)


def _device(p, bps=0):
    import torch
    t = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    mesh = bief.Mesh(p["ik"], p["x"].size)
    mesh.set_blocks_per_sm(bps)
    A = bief.Matrix(mesh)
    A.assemble_wave(t(p["x"]), t(p["y"]), t(p["coef"]))
    return mesh, A, t


def test_1m_assembly_and_matvec_bitexact(wave1m):
    import torch
    mesh, A, t = _device(wave1m)
    dm, xm, td = A.get()
    assert td == "Q"
    assert np.array_equal(dm, wave1m["dm"]) and np.array_equal(xm, wave1m["xm"])
    out = torch.zeros(dm.size, dtype=torch.float64, device="cuda")
    bief.matvec("X=AY    ", out, A, t(wave1m["xt"]))
    np.testing.assert_array_equal(out.cpu().numpy(), wave1m["b"])
    mesh.close()


@pytest.mark.parametrize("bps", [1, 2])
def test_1m_fp64_gracjg_bitexact(oracle_mod, wave1m, bps):
    import torch
    mesh, A, t = _device(wave1m, bps)
    x = torch.zeros(wave1m["x"].size, dtype=torch.float64, device="cuda")
    cfg = bief.SlvCfg(slv=1, nitmax=1000000, precon=2, krylov=0, eps=1e-8, zero=0.0)
    st, nit, relres = bief.solve(x, A, t(wave1m["b"]), cfg)
    G, T = mesh.launch_info()
    with oracle_mod.threads():
        r = oracle_mod.solve(wave1m["ik"], wave1m["dm"], "Q", wave1m["xm"], "S", wave1m["b"],
                             eps=1e-8, nitmax=1000000, dot_mode=oracle_mod.DOT_BLOCKED,
                             nblocks=G, nthreads=T)
    assert st == r["status"] == 0
    assert nit == r["nit"] and relres == r["relres"] and relres <= 1e-8
    np.testing.assert_array_equal(x.cpu().numpy(), r["x"])
    mesh.close()


@pytest.mark.parametrize("bps", [1, 2])
def test_1m_mixed_bitexact(oracle_mod, wave1m, bps):
    import torch
    mesh, A, t = _device(wave1m, bps)
    x = torch.zeros(wave1m["x"].size, dtype=torch.float64, device="cuda")
    st, outer, inner, relres = bief.solve_mixed(x, A, t(wave1m["b"]), precon=2, inner_tol=0.1,
                                                outer_tol=1e-8)
    G, T = mesh.launch_info()
    with oracle_mod.threads():
        r = oracle_mod.solve_mixed(wave1m["ik"], wave1m["dm"], "Q", wave1m["xm"], wave1m["b"],
                                   precon=2, inner_tol=0.1, outer_tol=1e-8, max_outer=1000,
                                   max_inner=1000000, nblocks=G, nthreads=T)
    assert st == r["status"] == 0
    assert (outer, inner) == (r["outer"], r["inner"])
    assert relres == r["relres"] and relres <= 1e-8
    np.testing.assert_array_equal(x.cpu().numpy(), r["x"])
    mesh.close()


@pytest.mark.parametrize("npt,tpb", [(8, 1024), (4, 256)])
def test_batch256_instances_bitexact(oracle_mod, npt, tpb):
    """The batch workload itself (256 meshes, 13.0M nodes), tile shapes the
    autotuner picks from: every instance converges, and the smallest, the
    median and the largest equal the oracle bit for bit."""
    import torch
    from opentelemac_b200.batch import BatchSolver
    sizes = mg.batch_sizes()
    inst = [mg.batch_instance(k, n) for k, n in enumerate(sizes)]
    bs = BatchSolver([(x.size, ik) for x, y, ik, coef, b in inst])
    bs.assemble_wave([v[0] for v in inst], [v[1] for v in inst], [v[3] for v in inst])
    b = bs.gather([v[4] for v in inst])
    x = torch.zeros_like(b)
    r = bs.solve_mixed(x, b, inner_tol=1e-4, outer_tol=1e-8, nodes_per_thread=npt,
                       threads_per_block=tpb)
    assert (r["status"] == 0).all() and (r["relres"] <= 1e-8).all()
    xs = bs.scatter(x)
    order = np.argsort([v[0].size for v in inst], kind="stable")
    for k in (order[0], order[len(order) // 2], order[-1]):
        xk, yk, ik, coef, bk = inst[k]
        dm, xm = oracle_mod.wave_matrix(xk, yk, ik, coef)
        with oracle_mod.threads():
            ref = oracle_mod.solve_mixed_batch(ik, dm, "Q", xm, bk, precon=2, inner_tol=1e-4,
                                               outer_tol=1e-8, nthreads=tpb, npt=npt)
        assert ref["status"] == 0
        assert (r["inner"][k], r["outer"][k]) == (ref["inner"], ref["outer"]), k
        assert r["relres"][k] == ref["relres"]
        np.testing.assert_array_equal(xs[k].cpu().numpy(), ref["x"], err_msg=f"instance {k}")
    bs.close()
