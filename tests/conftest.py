import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


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
