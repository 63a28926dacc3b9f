"""Generate the golden fixtures under tests/golden/.

The reference (Fortran) cannot be built in this environment and ships no
solver-level golden vectors, so these fixtures are produced by the C oracle
(oracle/bief_oracle.c, a line-by-line restatement of the reference
routines).  They freeze the oracle's outputs so that the oracle itself and
the device kernels are checked against fixed numbers.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from opentelemac_b200 import meshgen as mg  # noqa: E402


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def problem(n, field):
    x, y, ik = mg.square_mesh(n)
    h = mg.depth_smooth(x, y, ik) if field == "smooth" else mg.depth_loguniform(ik)
    coef = mg.wave_coef(h)
    dm, xm = oracle.wave_matrix(x, y, ik, coef)
    xt = mg.random_solution(x.size)
    b = oracle.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    return x, y, ik, coef, dm, xm, xt, b


def main():
    oracle.build()
    # 21 x 21: everything stored
    x, y, ik, coef, dm, xm, xt, b = problem(21, "smooth")
    out = dict(x=x, y=y, ikle0=ik, coef=coef, dm=dm, xm=xm, xt=xt, b=b)
    for nit in (1, 10):
        r = oracle.solve(ik, dm, "Q", xm, "S", b, precon=2, nitmax=nit, eps=1e-30)
        out[f"x_nit{nit}"] = r["x"]
        # the device's dot order for a mesh this size: 1 block of 1024 threads
        r = oracle.solve(ik, dm, "Q", xm, "S", b, precon=2, nitmax=nit, eps=1e-30,
                         dot_mode=oracle.DOT_BLOCKED, nblocks=1, nthreads=1024)
        out[f"x_nit{nit}_blocked"] = r["x"]
    r = oracle.solve(ik, dm, "Q", xm, "S", b, precon=2, nitmax=100000, eps=1e-8)
    out.update(x_final=r["x"], nit_final=r["nit"], relres_final=r["relres"],
               b_scaled=r["b"], xm_scaled=r["xm"], dm_scaled=r["dm"])
    rb = oracle.solve(ik, dm, "Q", xm, "S", b, precon=2, nitmax=100000, eps=1e-8,
                      dot_mode=oracle.DOT_BLOCKED, nblocks=1, nthreads=1024)
    out.update(x_final_blocked=rb["x"], nit_final_blocked=rb["nit"])
    for op in ("X=AY    ", "X=TAY   "):
        out["mv_" + op.strip().replace("=", "")] = oracle.matvec(op, ik, dm, "Q", xm, "S", xt)
    np.savez_compressed(os.path.join(HERE, "golden_21.npz"), **out)

    # 101 x 101 (config 0 construction): digests of the inputs, solution
    x, y, ik, coef, dm, xm, xt, b = problem(101, "smooth")
    r = oracle.solve(ik, dm, "Q", xm, "S", b, precon=2, nitmax=100000, eps=1e-8)
    np.savez_compressed(
        os.path.join(HERE, "golden_101.npz"),
        mesh_digest=digest(x, y, ik), matrix_digest=digest(dm, xm), b_digest=digest(b),
        x_final=r["x"], nit_final=r["nit"], relres_final=r["relres"])
    print("wrote golden_21.npz, golden_101.npz")


if __name__ == "__main__":
    main()
