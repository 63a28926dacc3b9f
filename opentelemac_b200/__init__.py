"""opentelemac_b200 -- B200-native (sm_100a) drop-in for TELEMAC-MASCARET
BIEF's element-by-element P1 conjugate-gradient solve (SOLVE -> GRACJG,
MATVEC -> MV0303 + ASSVEC).

    from opentelemac_b200 import bief, meshgen
    mesh = bief.Mesh(ikle0, npoin)
    A = bief.Matrix(mesh, dm, xm, "Q", "S")
    cfg = bief.SlvCfg(slv=1, nitmax=100000, precon=2, eps=1e-8)
    status, nit, relres = bief.solve(x, A, b, cfg)
"""
from . import meshgen  # noqa: F401

__all__ = ["bief", "meshgen", "autograd", "batch"]
