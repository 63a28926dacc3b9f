"""The restatement on several host threads gives the same bits as on one.

The large-case parity tests (1M nodes, the 256-mesh batch) run the oracle
with OpenMP so that it finishes in seconds; what makes that legitimate is
that only loops with independent iterations are shared out, and the
binary64 MATVEC inside the threaded solves is the per-node gather form of
MV0303 + ASSVEC.  These checks run both forms on meshes above the threading
threshold and compare every bit."""
import numpy as np
import pytest

from conftest import small_problem


@pytest.fixture
def threaded(oracle_mod):
    yield oracle_mod.threads(4)
    oracle_mod.set_threads(1)


@pytest.mark.parametrize("shuffle,field", [(False, "smooth"), (True, "loguniform")])
def test_threaded_solve_blocked_same_bits(oracle_mod, threaded, shuffle, field):
    p = small_problem(oracle_mod, n=121, shuffle=shuffle, field=field)
    args = (p["ik"], p["dm"], "Q", p["xm"], "S", p["b"])
    kw = dict(precon=2, eps=1e-9, dot_mode=oracle_mod.DOT_BLOCKED, nblocks=13, nthreads=256)
    ref = oracle_mod.solve(*args, **kw)
    with threaded:
        got = oracle_mod.solve(*args, **kw)
    assert ref["status"] == got["status"] == 0
    assert ref["nit"] == got["nit"] and ref["relres"] == got["relres"]
    for k in ("x", "b", "dm", "xm"):
        assert np.array_equal(ref[k], got[k]), k


def test_threaded_solve_sequential_dots_same_bits(oracle_mod, threaded):
    """The reference's own sequential dot order stays sequential; the
    gather MATVEC and the threaded vector updates leave the bits as they
    are, also for TYPDIA 'I' and PRECON 1 (no change of variables)."""
    p = small_problem(oracle_mod, n=101)
    for precon, typdia in ((2, "Q"), (1, "I"), (5, "Q")):
        args = (p["ik"], p["dm"], typdia, p["xm"], "S", p["b"])
        ref = oracle_mod.solve(*args, precon=precon, eps=1e-8, nitmax=300)
        with threaded:
            got = oracle_mod.solve(*args, precon=precon, eps=1e-8, nitmax=300)
        assert ref["nit"] == got["nit"] and ref["relres"] == got["relres"]
        assert np.array_equal(ref["x"], got["x"])


@pytest.mark.parametrize("npt,nt", [(1, 1024), (4, 256)])
def test_threaded_mixed_same_bits(oracle_mod, threaded, npt, nt):
    p = small_problem(oracle_mod, n=111, field="loguniform")
    args = (p["ik"], p["dm"], "Q", p["xm"], p["b"])
    ref = oracle_mod.solve_mixed(*args, inner_tol=1e-4, outer_tol=1e-9, nblocks=9, nthreads=nt)
    refb = oracle_mod.solve_mixed_batch(*args, inner_tol=1e-4, outer_tol=1e-9, nthreads=nt,
                                        npt=npt)
    with threaded:
        got = oracle_mod.solve_mixed(*args, inner_tol=1e-4, outer_tol=1e-9, nblocks=9,
                                     nthreads=nt)
        gotb = oracle_mod.solve_mixed_batch(*args, inner_tol=1e-4, outer_tol=1e-9, nthreads=nt,
                                            npt=npt)
    for r, g in ((ref, got), (refb, gotb)):
        assert r["status"] == g["status"] == 0
        assert (r["inner"], r["outer"], r["relres"]) == (g["inner"], g["outer"], g["relres"])
        assert np.array_equal(r["x"], g["x"])


def test_threaded_dots_same_bits(oracle_mod, threaded):
    rng = np.random.default_rng(3)
    for n in (4096, 40000, 1002001):
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        ref = [oracle_mod.dot(x, y, oracle_mod.DOT_BLOCKED, 148, 1024),
               oracle_mod.dot_batch(x, y, 1024, 8), oracle_mod.dot_batch(x, y, 256, 1)]
        with threaded:
            got = [oracle_mod.dot(x, y, oracle_mod.DOT_BLOCKED, 148, 1024),
                   oracle_mod.dot_batch(x, y, 1024, 8), oracle_mod.dot_batch(x, y, 256, 1)]
        assert ref == got
