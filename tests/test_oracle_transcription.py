"""A second, independent restatement of SOLVE(SLV=1, PRECON=2) in plain
Python, checked bit for bit against the C oracle.

The C oracle is the checker for every device test, so an error in it would
pass unseen wherever the device copies it.  This file restates the same
Fortran a second time, statement by statement, with Python floats (IEEE
binary64, every operation rounded, no fused multiply-add) and plain loops in
the reference's loop order, and requires the C oracle's sequential-dot mode
to give the same bits: iteration count, residual, solution, and the
side effects SOLVE leaves on B and on the matrix.  The matrix builder the
parity cases share (mass plus P0 diffusion) is restated the same way.

The reference statements followed:
  solve.f:480-497      PREXSM = .TRUE., DIADON = .FALSE., PRECDT -> PRECD1
  precd1.f             D = A%D; D = SQRT(D); X = X*D; D = 1/D (OVD IOPT 2,
                       EPS 1e-10, value 1); OM('M=DMD'); TYPDIA = 'I';
                       B = B*D
  om1111.f:559-580     DMD for TYPDIA 'Q' (DM*D twice) and TYPEXT 'S'
                       (XM(e,k) * D(second node) * D(first node))
  solve.f:465-476      IG = IT5: with diagonal preconditioning G and R are
                       the same array in GRACJG
  gracjg.F:60-168      the iteration, PREC false
  matvct.f:279-292     MV0303 with the symmetric pointers
                       XA21 = XA12, XA31 = XA13, XA32 = XA23
  mv0303.f:117-157     W1..W3 per element, then X = Y*DA (or X = Y for 'I')
  matvct.f:552-558     ASSVEC with INIT .FALSE.: IDP = 1..3, elements in order
  assve1.f             X(IKLE(E)) = X(IKLE(E)) + W(E)
  dot.f                DOT = DOT + X(I)*Y(I), I = 1..NPOIN
  ov.f:196,292,316,324 X*Y, X-Y, Y+C*Z, X+C*Y
  solve.f:636-641      X = X*D after the solver
"""
import math

import numpy as np
import pytest

from conftest import small_problem

RMIN = 1.0e-15  # gracjg.F:97


def _dot(x, y):
    s = 0.0
    for i in range(len(x)):
        s = s + x[i] * y[i]
    return s


def _matvec_x_ay(ikle, da, typdia, xa12, xa13, xa23, y):
    """MATVEC('X=AY    ') on an EBE P1 matrix, TYPEXT 'S'."""
    ne = len(ikle)
    w1, w2, w3 = [0.0] * ne, [0.0] * ne, [0.0] * ne
    for e in range(ne):
        i1, i2, i3 = ikle[e]
        w1[e] = xa12[e] * y[i2] + xa13[e] * y[i3]
        w2[e] = xa23[e] * y[i3] + xa12[e] * y[i1]
        w3[e] = xa13[e] * y[i1] + xa23[e] * y[i2]
    if typdia == "Q":
        x = [y[i] * da[i] for i in range(len(y))]
    elif typdia == "I":
        x = list(y)
    else:
        x = [0.0] * len(y)
    for k, w in enumerate((w1, w2, w3)):
        for e in range(ne):
            j = ikle[e][k]
            x[j] = x[j] + w[e]
    return x


def _solve_cg_diag(ikle, dm, xm, b, x, eps, nitmax):
    """SOLVE with SLV=1, PRECON=2, TYPDIA 'Q', TYPEXT 'S', MODASS=1, one
    process.  Works on Python lists; returns everything SOLVE leaves."""
    n = len(b)
    ne = len(ikle)
    xa12, xa13, xa23 = list(xm[0]), list(xm[1]), list(xm[2])
    dm, b, x = list(dm), list(b), list(x)

    # PRECD1
    d = list(dm)
    d = [math.sqrt(v) for v in d]
    x = [x[i] * d[i] for i in range(n)]
    d = [1.0 / v if abs(v) > 1.0e-10 else 1.0 for v in d]
    dm = [dm[i] * d[i] for i in range(n)]
    dm = [dm[i] * d[i] for i in range(n)]
    for e in range(ne):
        i1, i2, i3 = ikle[e]
        xa12[e] = xa12[e] * d[i2] * d[i1]
        xa13[e] = xa13[e] * d[i3] * d[i1]
        xa23[e] = xa23[e] * d[i3] * d[i2]
    typdia = "I"
    b = [b[i] * d[i] for i in range(n)]

    def av(v):
        return _matvec_x_ay(ikle, dm, typdia, xa12, xa13, xa23, v)

    # GRACJG, G and R the same array
    m = 0
    status = 0
    xl = _dot(b, b)
    if math.sqrt(xl) < RMIN:
        x = [0.0] * n
        rmrm = 0.0
        xl = 1.0
    else:
        if xl < 1.0:
            xl = 1.0
        r = av(x)
        r = [r[i] - b[i] for i in range(n)]
        rmrm = _dot(r, r)
        rmgm = rmrm
        if not rmrm < eps * eps * xl:
            dd = list(r)
            ad = av(dd)
            dad = _dot(dd, ad)
            ro = rmgm / dad
            x = [x[i] + (-ro) * dd[i] for i in range(n)]
            while True:
                m = m + 1
                r = [r[i] + (-ro) * ad[i] for i in range(n)]
                rm1gm1 = rmgm
                rmrm = _dot(r, r)
                rmdm = rmrm
                rmgm = rmrm
                if rmrm <= xl * (eps * eps):
                    break
                beta = rmgm / rm1gm1
                dd = [r[i] + beta * dd[i] for i in range(n)]
                ad = av(dd)
                dad = _dot(dd, ad)
                ro = rmdm / dad
                x = [x[i] + (-ro) * dd[i] for i in range(n)]
                if not m < nitmax:
                    status = 1
                    break

    # back to the unscaled unknown
    x = [x[i] * d[i] for i in range(n)]
    return dict(x=np.array(x), b=np.array(b), dm=np.array(dm),
                xm=np.array([xa12, xa13, xa23]), typdia=typdia, nit=m, status=status,
                relres=math.sqrt(rmrm / xl))


def _ikle_rows(ik):
    ik = np.asarray(ik)
    if ik.shape[0] == 3 and ik.shape[1] != 3:
        ik = ik.T
    return [tuple(int(v) for v in row) for row in ik]


CASES = [
    dict(n=21, shuffle=False, field="smooth", seed=12345, eps=1e-8, x0=False),
    dict(n=21, shuffle=True, field="loguniform", seed=7, eps=1e-10, x0=True),
    dict(n=31, shuffle=True, field="smooth", seed=99, eps=1e-9, x0=False),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "n%d_%s_%s" % (
    c["n"], c["field"], "shuf" if c["shuffle"] else "plain"))
def test_transcription_equals_c_oracle(oracle_mod, case):
    p = small_problem(oracle_mod, n=case["n"], shuffle=case["shuffle"],
                      field=case["field"], seed=case["seed"])
    n = p["b"].size
    ikle = _ikle_rows(p["ik"])
    ne = len(ikle)
    xm = np.asarray(p["xm"], dtype=np.float64).reshape(-1, ne)
    x0 = (np.random.default_rng(case["seed"]).standard_normal(n) if case["x0"]
          else np.zeros(n))

    py = _solve_cg_diag(ikle, p["dm"], xm, p["b"], x0, case["eps"], 100000)
    c = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", p["b"], x0=x0,
                         eps=case["eps"], dot_mode=oracle_mod.DOT_SEQUENTIAL)

    assert py["status"] == 0 and c["status"] == 0
    assert py["nit"] == c["nit"] and py["nit"] > 5
    assert py["relres"] == c["relres"]
    assert np.array_equal(py["x"], c["x"])
    assert np.array_equal(py["b"], c["b"])
    assert np.array_equal(py["dm"], c["dm"])
    assert np.array_equal(py["xm"], np.asarray(c["xm"]).reshape(-1, ne))
    assert py["typdia"] == c["typdia"] == "I"
    # and the answer is the one b was made from
    assert np.linalg.norm(py["x"] - p["xt"]) / np.linalg.norm(p["xt"]) < 1e-5


def test_transcription_matvec_equals_c_oracle(oracle_mod):
    """MATVEC('X=AY    ') alone, both diagonal types."""
    p = small_problem(oracle_mod, n=21, shuffle=True, field="loguniform", seed=3)
    ikle = _ikle_rows(p["ik"])
    ne = len(ikle)
    xm = np.asarray(p["xm"], dtype=np.float64).reshape(-1, ne)
    y = np.random.default_rng(5).standard_normal(p["b"].size)
    for typdia in ("Q", "I"):
        py = _matvec_x_ay(ikle, list(p["dm"]), typdia, list(xm[0]), list(xm[1]),
                          list(xm[2]), list(y))
        c = oracle_mod.matvec("X=AY    ", p["ik"], p["dm"], typdia, p["xm"], "S", y)
        assert np.array_equal(np.array(py), c)


def _wave_matrix(x, y, ikle, coef):
    """AM1 as PROPAG builds it: MATRIX('M=N', mass, XMUL 1) then
    MATRIX('M=M+N', diffusion with the P0 viscosity coef, XMUL 1).
      inbief.f:369-391  XEL, YEL relative to the element's first node
      surv11.f          SURFAC = 0.5*(X2*Y3 - X3*Y2)
      mt01aa.f          DET = SURFAC*(XMUL/12); off-diagonals DET, diagonal DET+DET
      mt02aa.f:106-144  P0 isotropic viscosity
      assvec.f          each MATRIX call assembles its own diagonal (INIT .TRUE.)
      om1111.f          'M=M+N': DM = DM + DN, XM = XM + XN column by column"""
    ne = len(ikle)
    dm = [0.0] * len(x)
    dn = [0.0] * len(x)
    xm = [[0.0] * ne for _ in range(3)]
    xn = [[0.0] * ne for _ in range(3)]
    m11, m22, m33 = [0.0] * ne, [0.0] * ne, [0.0] * ne
    n11, n22, n33 = [0.0] * ne, [0.0] * ne, [0.0] * ne
    sur12 = 1.0 / 12.0
    for e in range(ne):
        i1, i2, i3 = ikle[e]
        x2 = x[i2] - x[i1]
        x3 = x[i3] - x[i1]
        y2 = y[i2] - y[i1]
        y3 = y[i3] - y[i1]
        surfac = 0.5 * (x2 * y3 - x3 * y2)
        det = surfac * sur12
        xm[0][e] = det
        xm[1][e] = det
        xm[2][e] = det
        m11[e] = det + det
        m22[e] = det + det
        m33[e] = det + det
        s2d = 1.0 * 0.25 / surfac
        visc1 = coef[e] * s2d
        # Y3**2 with an integer exponent is Y3*Y3 in Fortran; Python's
        # float ** calls libm pow, which is not always the rounded product
        bpe = visc1 * (y3 * y3 + x3 * x3)
        cpf = visc1 * (y2 * y3 + x2 * x3)
        apd = visc1 * (y2 * y2 + x2 * x2)
        n11[e] = apd + bpe - 2 * cpf
        n22[e] = bpe
        n33[e] = apd
        xn[0][e] = cpf - bpe
        xn[1][e] = cpf - apd
        xn[2][e] = -cpf
    for k, w in enumerate((m11, m22, m33)):
        for e in range(ne):
            j = ikle[e][k]
            dm[j] = dm[j] + w[e]
    for k, w in enumerate((n11, n22, n33)):
        for e in range(ne):
            j = ikle[e][k]
            dn[j] = dn[j] + w[e]
    dm = [dm[i] + dn[i] for i in range(len(x))]
    xm = [[xm[k][e] + xn[k][e] for e in range(ne)] for k in range(3)]
    return np.array(dm), np.array(xm)


@pytest.mark.parametrize("shuffle,field", [(False, "smooth"), (True, "loguniform")])
def test_transcription_wave_matrix_equals_c_oracle(oracle_mod, shuffle, field):
    """The matrix every parity case is built on, restated from the same
    element routines."""
    p = small_problem(oracle_mod, n=21, shuffle=shuffle, field=field, seed=11)
    ikle = _ikle_rows(p["ik"])
    dm, xm = _wave_matrix([float(v) for v in p["x"]], [float(v) for v in p["y"]], ikle,
                          [float(v) for v in p["coef"]])
    assert np.array_equal(dm, p["dm"])
    assert np.array_equal(xm, np.asarray(p["xm"]).reshape(-1, len(ikle)))


def test_transcription_zero_rhs(oracle_mod):
    """B = 0: GRACJG's RMIN branch sets X = 0 and does no iteration."""
    p = small_problem(oracle_mod, n=21)
    n = p["b"].size
    ikle = _ikle_rows(p["ik"])
    xm = np.asarray(p["xm"], dtype=np.float64).reshape(-1, len(ikle))
    x0 = np.ones(n)
    py = _solve_cg_diag(ikle, p["dm"], xm, np.zeros(n), x0, 1e-8, 100)
    c = oracle_mod.solve(p["ik"], p["dm"], "Q", p["xm"], "S", np.zeros(n), x0=x0, eps=1e-8)
    assert py["nit"] == c["nit"] == 0
    assert np.array_equal(py["x"], c["x"]) and not py["x"].any()


def test_transcription_on_the_gouttedo_mesh(oracle_mod):
    """The reference's own gouttedo mesh (4,624 nodes, its node and element
    numbering as drawn, frozen in tests/golden/gouttedo.npz): the matrix
    build, MATVEC and 40 GRACJG iterations of the two restatements agree
    bit for bit."""
    from conftest import gouttedo_mesh
    from opentelemac_b200 import meshgen as mg
    gx, gy, ik, _ = gouttedo_mesh()
    npoin = gx.size
    ikle = _ikle_rows(ik)
    x = [float(v) for v in gx]
    y = [float(v) for v in gy]
    coef = mg.wave_coef(mg.depth_smooth(gx, gy, ik))
    dm, xm = _wave_matrix(x, y, ikle, [float(v) for v in coef])
    cdm, cxm = oracle_mod.wave_matrix(gx, gy, ik, coef)
    assert np.array_equal(dm, cdm)
    assert np.array_equal(xm, np.asarray(cxm).reshape(3, -1))
    xt = mg.random_solution(npoin)
    b = _matvec_x_ay(ikle, list(dm), "Q", list(xm[0]), list(xm[1]), list(xm[2]), list(xt))
    cb = oracle_mod.matvec("X=AY    ", ik, cdm, "Q", cxm, "S", xt)
    assert np.array_equal(np.array(b), cb)
    py = _solve_cg_diag(ikle, dm, xm, cb, np.zeros(npoin), 1e-12, 40)
    c = oracle_mod.solve(ik, cdm, "Q", cxm, "S", cb, eps=1e-12, nitmax=40,
                         dot_mode=oracle_mod.DOT_SEQUENTIAL)
    assert py["status"] == 1 and c["status"] != 0
    assert py["nit"] == c["nit"] == 40
    assert py["relres"] == c["relres"]
    assert np.array_equal(py["x"], c["x"])
