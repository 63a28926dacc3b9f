"""SERAFIN (.slf) mesh and result files: write/read round trips, the
reference's own example files when the reference tree is present, and a
mesh read from a file carried through the segment numbering and the
oracle's solve."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, REFERENCE
from opentelemac_b200 import meshgen as mg, serafin

# the reference's TELEMAC-2D examples, where TELEMAC_REFERENCE names its tree
REF_EXAMPLES = os.path.join(REFERENCE, "examples", "telemac2d") if REFERENCE else ""


@pytest.mark.parametrize("double", [False, True])
@pytest.mark.parametrize("endian", [">", "<"])
def test_round_trip(tmp_path, double, endian):
    x, y, ik = mg.delaunay_mesh(500)
    rng = np.random.default_rng(1)
    frames = [rng.uniform(-1, 1, (2, x.size)) for _ in range(3)]
    s = serafin.Serafin(title="round trip", var_names=["WATER DEPTH", "FREE SURFACE"],
                        var_units=["M", "M"], ikle=ik, x=x, y=y, times=[0.0, 0.5, 1.0],
                        values=frames, double=double, endian=endian,
                        date=[2024, 1, 2, 3, 4, 5])
    p = tmp_path / "m.slf"
    serafin.write(p, s)
    r = serafin.read(p)
    assert r.endian == endian and r.double == double
    assert r.title.endswith("SERAFIND" if double else "SERAFIN ")
    assert r.var_names == ["WATER DEPTH", "FREE SURFACE"] and r.var_units == ["M", "M"]
    np.testing.assert_array_equal(r.ikle, ik)
    np.testing.assert_array_equal(r.date, [2024, 1, 2, 3, 4, 5])
    cast = (lambda a: a) if double else (lambda a: np.asarray(a, np.float32).astype(np.float64))
    np.testing.assert_array_equal(r.x, cast(x))
    np.testing.assert_array_equal(r.y, cast(y))
    assert r.times == [0.0, 0.5, 1.0]
    for a, b in zip(r.values, frames):
        np.testing.assert_array_equal(a, cast(b))
    # and a rewrite reproduces the same bytes
    q = tmp_path / "m2.slf"
    serafin.write(q, r)
    assert open(p, "rb").read() == open(q, "rb").read()


def test_truncated_file_rejected(tmp_path):
    x, y, ik = mg.square_mesh(5)
    p = tmp_path / "t.slf"
    serafin.mesh_file(p, x, y, ik)
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-10])
    with pytest.raises(ValueError):
        serafin.read(p)


@pytest.mark.skipif(not REF_EXAMPLES or not os.path.isdir(REF_EXAMPLES),
                    reason="TELEMAC_REFERENCE not set to the reference tree")
def test_reference_example_files(oracle_mod, tmp_path):
    files = sorted(glob.glob(os.path.join(REF_EXAMPLES, "*", "geo*.slf")))[:40]
    assert files
    for f in files:
        s = serafin.read(f, values=False)
        assert s.ikle.min() >= 0 and s.ikle.max() < s.npoin
    # a result file with time steps, rewritten byte for byte (the file may
    # carry trailing bytes after its last record)
    f = os.path.join(REF_EXAMPLES, "gouttedo", "f2d_gouttedo.slf")
    s = serafin.read(f)
    assert len(s.times) == 21 and s.var_names[-1] == "WATER DEPTH"
    tmp = tmp_path / "rt.slf"
    serafin.write(tmp, s)
    a, b = open(f, "rb").read(), open(tmp, "rb").read()
    assert a[:len(b)] == b and len(a) - len(b) < 8
    # the real mesh through the segment numbering and the oracle's solve
    ik = s.ikle.astype(np.int32)
    g = mg.segments(ik, s.npoin)
    be, bf = mg.boundary_faces(ik)
    o = oracle_mod.stoseg(ik, s.npoin, be, bf)
    for p_, q_ in zip(g, o):
        np.testing.assert_array_equal(p_, q_)
    dm, xm = oracle_mod.wave_matrix(s.x, s.y, ik, mg.wave_coef(mg.depth_smooth(s.x, s.y, ik)))
    b = oracle_mod.matvec("X=AY    ", ik, dm, "Q", xm, "S", mg.random_solution(s.npoin))
    r = oracle_mod.solve(ik, dm, "Q", xm, "S", b, eps=1e-10)
    assert r["status"] == 0 and r["relres"] <= 1e-10


@pytest.mark.skipif(not REF_EXAMPLES or not os.path.isdir(REF_EXAMPLES),
                    reason="TELEMAC_REFERENCE not set to the reference tree")
def test_gouttedo_fixture_is_the_reference_mesh():
    """tests/golden/gouttedo.npz holds the reference's geo_gouttedo.slf and
    geo_gouttedo.cli as they are (same file hashes, same mesh)."""
    import hashlib
    d = np.load(os.path.join(GOLDEN, "gouttedo.npz"))
    case = os.path.join(REF_EXAMPLES, "gouttedo")
    for name, key in (("geo_gouttedo.slf", "slf_sha256"), ("geo_gouttedo.cli", "cli_sha256")):
        with open(os.path.join(case, name), "rb") as fh:
            assert hashlib.sha256(fh.read()).hexdigest() == str(d[key])
    s = serafin.read(os.path.join(case, "geo_gouttedo.slf"), values=False)
    np.testing.assert_array_equal(s.x, d["x"])
    np.testing.assert_array_equal(s.y, d["y"])
    np.testing.assert_array_equal(s.ikle, d["ikle0"])


def test_gouttedo_fixture_mesh_is_valid():
    """The frozen mesh: 4,624 nodes, 8,978 counter-clockwise triangles,
    every node used, 268 boundary points that are exactly the nodes on
    boundary faces."""
    from conftest import gouttedo_mesh
    x, y, ik, nbor = gouttedo_mesh()
    assert x.size == 4624 and ik.shape == (8978, 3)
    assert np.array_equal(np.unique(ik), np.arange(x.size))
    a = (x[ik[:, 1]] - x[ik[:, 0]]) * (y[ik[:, 2]] - y[ik[:, 0]]) - \
        (x[ik[:, 2]] - x[ik[:, 0]]) * (y[ik[:, 1]] - y[ik[:, 0]])
    assert (a > 0).all()
    be, bf = mg.boundary_faces(ik)
    on_boundary = np.unique(ik[be, bf])
    assert nbor.size == 268
    np.testing.assert_array_equal(np.sort(nbor), on_boundary)
