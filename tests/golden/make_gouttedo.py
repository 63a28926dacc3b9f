"""Freeze the reference's gouttedo mesh into tests/golden/gouttedo.npz.

The TELEMAC-2D example `examples/telemac2d/gouttedo` (a drop of water in a
square basin) is the reference case closest to this path: its steering
file `t2d_gouttedo_reprod.cas` runs the wave equation
(TREATMENT OF THE LINEAR SYSTEM 2) with EBE storage (MATRIX STORAGE 1),
conjugate gradient (SOLVER 1), no preconditioning (PRECONDITIONING 0),
compensated assembly and dot products (FINITE ELEMENT ASSEMBLY 3),
SOLVER ACCURACY 1e-4, at most 100 iterations, TIME STEP 0.04, implicitation
0.6 for depth and velocity.  Its mesh `geo_gouttedo.slf` has 4,624 nodes
and 8,978 triangles in the reference's own node and element numbering.

This script copies that mesh (coordinates as stored, binary32 values widened
to binary64; IKLE 0-based; IPOBO) and the boundary numbering of
`geo_gouttedo.cli` (NBOR, column 12, 0-based here; LIHBOR, column 1) into a
fixture, so that the tests can run on the reference's own mesh wherever the
reference tree is absent.  The SHA-256 of both source files is stored with
it.

    TELEMAC_REFERENCE=<root of the TELEMAC-MASCARET tree> \
        python tests/golden/make_gouttedo.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from opentelemac_b200 import serafin  # noqa: E402

CASE = os.path.join("examples", "telemac2d", "gouttedo")


def sha256(path):
    with open(path, "rb") as fh:
        return hashlib.sha256(fh.read()).hexdigest()


def read_cli(path):
    """LIHBOR (column 1) and NBOR (column 12, 1-based) of a .cli file."""
    lihbor, nbor = [], []
    with open(path) as fh:
        for line in fh:
            f = line.split()
            if len(f) >= 12:
                lihbor.append(int(f[0]))
                nbor.append(int(f[11]))
    return np.array(lihbor, np.int32), np.array(nbor, np.int32)


def main():
    ref = os.environ.get("TELEMAC_REFERENCE")
    if not ref:
        sys.exit("set TELEMAC_REFERENCE to the root of the TELEMAC-MASCARET source tree")
    slf = os.path.join(ref, CASE, "geo_gouttedo.slf")
    cli = os.path.join(ref, CASE, "geo_gouttedo.cli")
    s = serafin.read(slf, values=False)
    lihbor, nbor = read_cli(cli)
    out = dict(x=s.x, y=s.y, ikle0=s.ikle.astype(np.int32), ipobo=s.ipobo.astype(np.int32),
               nbor0=nbor - 1, lihbor=lihbor, slf_sha256=sha256(slf), cli_sha256=sha256(cli),
               source=os.path.join(CASE, "geo_gouttedo.slf"))
    dst = os.path.join(HERE, "gouttedo.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst}: {s.npoin} nodes, {s.nelem} elements, {nbor.size} boundary points")


if __name__ == "__main__":
    main()
