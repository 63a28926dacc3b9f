import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# Root of the TELEMAC-MASCARET source tree, for the tests that read its
# example files directly (skipped when unset); the gouttedo mesh they need
# most is frozen in tests/golden/gouttedo.npz (tests/golden/make_gouttedo.py).
REFERENCE = os.environ.get("TELEMAC_REFERENCE", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cfg0_problem(oracle_mod):
    """Config 0: 101x101 nodes, smooth depth, b = A x_true."""
    from opentelemac_b200 import meshgen as mg
    x, y, ik = mg.square_mesh(101)
    coef = mg.wave_coef(mg.depth_smooth(x, y, ik))
    dm, xm = oracle_mod.wave_matrix(x, y, ik, coef)
    xt = mg.random_solution(x.size)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    return dict(x=x, y=y, ik=ik, coef=coef, dm=dm, xm=xm, xt=xt, b=b)


def small_problem(oracle_mod, n=21, shuffle=False, field="smooth", seed=12345):
    from opentelemac_b200 import meshgen as mg
    x, y, ik = mg.square_mesh(n, seed=seed)
    if shuffle:
        x, y, ik, _, _ = mg.shuffled(x, y, ik)
    h = mg.depth_smooth(x, y, ik) if field == "smooth" else mg.depth_loguniform(ik)
    coef = mg.wave_coef(h)
    dm, xm = oracle_mod.wave_matrix(x, y, ik, coef)
    xt = mg.random_solution(x.size)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    return dict(x=x, y=y, ik=ik, coef=coef, dm=dm, xm=xm, xt=xt, b=b)


@pytest.fixture
def rng():
    return np.random.default_rng(2024)


def gouttedo_mesh():
    """The reference's gouttedo mesh (examples/telemac2d/gouttedo,
    geo_gouttedo.slf: 4,624 nodes, 8,978 triangles, its own numbering) and
    its boundary points (geo_gouttedo.cli NBOR, 0-based)."""
    d = np.load(os.path.join(GOLDEN, "gouttedo.npz"))
    return d["x"], d["y"], d["ikle0"], d["nbor0"]


# The case's settings (t2d_gouttedo_reprod.cas): TIME STEP 0.04,
# IMPLICITATION FOR DEPTH / VELOCITY 0.6; SOLVER 1, PRECONDITIONING 0,
# SOLVER ACCURACY 1e-4, at most 100 iterations, FINITE ELEMENT ASSEMBLY 3.
GOUTTEDO_DT, GOUTTEDO_TETA, GRAV = 0.04, 0.6, 9.81


def gouttedo_problem(oracle_mod):
    """PROPAG's wave-equation operator on the gouttedo mesh at the first
    time step: AM1 = MATMAS/DT + MATDIFUV with XMUL = -1, U = DM1 and
    V = HPROP (propag.F:661-677,1397,1407-1408).  At rest the momentum
    matrix's diagonal is the nodal mass over DT, so DM1 = -TETAU TETAH GRAV
    DT; HPROP is the case's initial depth, the drop of its condin.f
    ('PARTICULAR': H = 2.4 (1 + exp(-((x-10.05)^2 + (y-10.05)^2)/4))).
    b = A x_true with a random x_true."""
    from opentelemac_b200 import meshgen as mg
    x, y, ik, nbor = gouttedo_mesh()
    h = 2.4 * (1.0 + np.exp(-((x - 10.05) * (x - 10.05) + (y - 10.05) * (y - 10.05)) / 4.0))
    dm1 = np.full(x.size, -GOUTTEDO_TETA * GOUTTEDO_TETA * GRAV * GOUTTEDO_DT)
    dm, xm = oracle_mod.mass_diff_matrix(x, y, ik, dm1, h, kind=12,
                                         xmul_mass=1.0 / GOUTTEDO_DT, xmul_dif=-1.0)
    xt = mg.random_solution(x.size)
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", xt)
    return dict(x=x, y=y, ik=ik, nbor=nbor, h=h, dm1=dm1, dm=dm, xm=xm, xt=xt, b=b)
