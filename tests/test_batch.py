"""Batched multi-mesh solve (one persistent launch, per-instance masks):
every instance bit-exact against the oracle's restatement of the same
algorithm in the batched dot order, plus the 256-mesh workload."""
import numpy as np
import pytest

from opentelemac_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _instances(sizes, seed0=100):
    import oracle
    out = []
    for k, n in enumerate(sizes):
        x, y, ik = mg.square_mesh(n, seed=seed0 + k)
        h = mg.depth_smooth(x, y, ik) if k % 2 == 0 else mg.depth_loguniform(ik, seed=seed0 + k)
        coef = mg.wave_coef(h)
        dm, xm = oracle.wave_matrix(x, y, ik, coef)
        b = np.random.default_rng(seed0 + k).uniform(-1, 1, x.size)
        out.append(dict(x=x, y=y, ik=ik, coef=coef, dm=dm, xm=xm, b=b))
    return out


@pytest.mark.parametrize("bps", [1, 2])
@pytest.mark.parametrize("npt,threads", [(1, 1024), (2, 1024), (4, 256), (2, 512)])
def test_batch_bitexact_per_instance(oracle_mod, npt, threads, bps):
    """Each tile shape with the kernel built for one and for two blocks per
    SM (the batched dot order depends on the tile shape only)."""
    from opentelemac_b200.batch import BatchSolver
    inst = _instances([7, 15, 23, 40, 57, 33])
    inst[3]["b"] = np.zeros_like(inst[3]["b"])               # b = 0: x = 0 at once
    bs = BatchSolver([(p["x"].size, p["ik"]) for p in inst])
    bs.mesh.set_blocks_per_sm(bps)
    bs.assemble_wave([p["x"] for p in inst], [p["y"] for p in inst], [p["coef"] for p in inst])
    b = bs.gather([p["b"] for p in inst])
    x = bs.gather([np.zeros(p["x"].size) for p in inst])
    r = bs.solve_mixed(x, b, inner_tol=1e-4, outer_tol=1e-9, nodes_per_thread=npt,
                       threads_per_block=threads)
    xs = [v.cpu().numpy() for v in bs.scatter(x)]
    for k, p in enumerate(inst):
        ref = oracle_mod.solve_mixed_batch(p["ik"], p["dm"], "Q", p["xm"], p["b"], precon=2,
                                           inner_tol=1e-4, outer_tol=1e-9, npt=npt,
                                           nthreads=threads)
        assert r["status"][k] == ref["status"] == 0
        assert (r["inner"][k], r["outer"][k]) == (ref["inner"], ref["outer"]), k
        assert r["relres"][k] == ref["relres"]
        np.testing.assert_array_equal(xs[k], ref["x"], err_msg=f"instance {k}")
    assert r["inner"][3] == 0 and not xs[3].any()
    bs.close()


@pytest.mark.parametrize("bps", [1, 2])
@pytest.mark.parametrize("npt,threads", [(1, 1024), (4, 256)])
def test_batch_segments_bitexact_per_instance(oracle_mod, npt, threads, bps):
    """Segment storage (MATRIX STORAGE 3, TELEMAC-2D's default): every
    instance's own STOSEG numbering, the EBE matrix converted by ASSEX3 on the
    device, each instance bit for bit the oracle's batched segment solve."""
    from opentelemac_b200.batch import BatchSolver
    inst = _instances([9, 17, 31, 26, 44])
    inst[2]["b"] = np.zeros_like(inst[2]["b"])
    bs = BatchSolver([(p["x"].size, p["ik"]) for p in inst])
    bs.mesh.set_blocks_per_sm(bps)
    bs.assemble_wave([p["x"] for p in inst], [p["y"] for p in inst], [p["coef"] for p in inst])
    segs = [mg.segments(p["ik"], p["x"].size) for p in inst]
    bs.set_segments([(g[0], g[1]) for g in segs]).to_segments()
    assert bs.A.storage == 3
    b = bs.gather([p["b"] for p in inst])
    x = bs.gather([np.zeros(p["x"].size) for p in inst])
    r = bs.solve_mixed(x, b, inner_tol=1e-4, outer_tol=1e-9, nodes_per_thread=npt,
                       threads_per_block=threads)
    xs = [v.cpu().numpy() for v in bs.scatter(x)]
    for k, (p, (g1, g2, es, ori)) in enumerate(zip(inst, segs)):
        xa = oracle_mod.assex3(es, ori, "S", p["xm"], g1.size)
        ref = oracle_mod.solve_mixed_batch_seg(g1, g2, p["dm"], "Q", xa, p["b"], precon=2,
                                               inner_tol=1e-4, outer_tol=1e-9, npt=npt,
                                               nthreads=threads)
        assert r["status"][k] == ref["status"] == 0
        assert (r["inner"][k], r["outer"][k]) == (ref["inner"], ref["outer"]), k
        assert r["relres"][k] == ref["relres"]
        np.testing.assert_array_equal(xs[k], ref["x"], err_msg=f"instance {k}")
    assert r["inner"][2] == 0 and not xs[2].any()
    bs.close()


def test_batch_256_meshes():
    """256 meshes, node counts log-uniform in [2,000, 200,000], each with its
    own depth field seed and random right-hand side, one launch, relres 1e-8."""
    import torch
    from opentelemac_b200.batch import BatchSolver
    sizes = mg.batch_sizes()
    meshes, xs, ys, coefs, bs_ = [], [], [], [], []
    for k, n in enumerate(sizes):
        x, y, ik, coef, bv = mg.batch_instance(k, n)
        meshes.append((x.size, ik))
        xs.append(x)
        ys.append(y)
        coefs.append(coef)
        bs_.append(bv)
    bs = BatchSolver(meshes)
    bs.assemble_wave(xs, ys, coefs)
    b = bs.gather(bs_)
    x = torch.zeros_like(b)
    r = bs.solve_mixed(x, b, inner_tol=1e-4, outer_tol=1e-8)
    assert (r["status"] == 0).all()
    assert (r["relres"] <= 1e-8).all()
    # independent residual check on the three smallest instances
    import oracle
    order = np.argsort([m[0] for m in meshes])[:3]
    xl = bs.scatter(x)
    for k in order:
        n, ik = meshes[k]
        dm, xm = oracle.wave_matrix(xs[k], ys[k], ik, coefs[k])
        res = bs_[k] - oracle.matvec("X=AY    ", ik, dm, "Q", xm, "S", xl[k].cpu().numpy())
        d = 1.0 / np.sqrt(dm)
        assert np.linalg.norm(res * d) / np.linalg.norm(bs_[k] * d) <= 1.01e-8
    bs.close()


def test_batch_slot_columns_32bit(oracle_mod):
    """A batch with one randomly renumbered 40,401-node instance, whose
    binary32 slots need 32-bit columns (some neighbour lies more than 32,767
    nodes away), beside small row-wise instances: every instance bit for bit
    the oracle's."""
    from opentelemac_b200.batch import BatchSolver
    inst = _instances([13, 29])
    x, y, ik = mg.square_mesh(201, seed=77)
    x, y, ik, _, _ = mg.shuffled(x, y, ik, seed=78)
    e = np.concatenate([ik[:, [0, 1]], ik[:, [1, 2]], ik[:, [2, 0]]])
    assert np.abs(e[:, 0].astype(np.int64) - e[:, 1]).max() > 32767
    coef = mg.wave_coef(mg.depth_loguniform(ik, seed=79))
    dm, xm = oracle_mod.wave_matrix(x, y, ik, coef)
    inst.insert(1, dict(x=x, y=y, ik=ik, coef=coef, dm=dm, xm=xm,
                        b=np.random.default_rng(80).uniform(-1, 1, x.size)))
    bs = BatchSolver([(p["x"].size, p["ik"]) for p in inst])
    bs.assemble_wave([p["x"] for p in inst], [p["y"] for p in inst], [p["coef"] for p in inst])
    b = bs.gather([p["b"] for p in inst])
    xb = bs.gather([np.zeros(p["x"].size) for p in inst])
    r = bs.solve_mixed(xb, b, inner_tol=1e-4, outer_tol=1e-9, nodes_per_thread=2,
                       threads_per_block=1024)
    xs = [v.cpu().numpy() for v in bs.scatter(xb)]
    for k, p in enumerate(inst):
        ref = oracle_mod.solve_mixed_batch(p["ik"], p["dm"], "Q", p["xm"], p["b"], precon=2,
                                           inner_tol=1e-4, outer_tol=1e-9, npt=2, nthreads=1024)
        assert r["status"][k] == ref["status"] == 0
        assert (r["inner"][k], r["outer"][k]) == (ref["inner"], ref["outer"]), k
        np.testing.assert_array_equal(xs[k], ref["x"], err_msg=f"instance {k}")
    bs.close()
