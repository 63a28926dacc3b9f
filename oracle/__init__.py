"""CPU oracle for the BIEF EBE P1 CG path -- TEST INFRASTRUCTURE ONLY.

A plain-C restatement (bief_oracle.c) of the reference Fortran routines
SOLVE/PRECD1/GRACJG/MATVEC/MV0303/ASSVEC/DOT and of the element matrices
MT01AA/MT02AA, loaded with ctypes.  Only the tests, the smoke check and the
benchmark's CPU-baseline leg use it; the product library never does.

Parity unpinned: the reference cannot be compiled here (Fortran, no
compiler) and ships no solver-level golden vectors; the restatement is
cross-checked against dense numpy / scipy computations instead.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libbief_oracle.so")

DOT_SEQUENTIAL = 0
DOT_BLOCKED = 1
DOT_COMP_SEQUENTIAL = 2      # MODASS = 3 (dot_comp.f), the reference's order
DOT_COMP_BLOCKED = 3         # MODASS = 3 in the device kernels' order

_lib = None


def build(force=False):
    src = os.path.join(HERE, "bief_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(src) > os.path.getmtime(LIB):
        subprocess.run(["make", "-s", "-B" if force else "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.POINTER
        d, i, c = ctypes.c_double, ctypes.c_int, ctypes.c_char
        pd, pi = P(d), P(i)
        L.orc_wave_matrix.argtypes = [i, i, pd, pd, pi, pi, pi, pd, pd, pd]
        L.orc_wave_matrix_parts.argtypes = [i, i, pd, pd, pi, pi, pi, pd]
        L.orc_mass_diff_matrix.argtypes = [i, i, pd, pd, pi, pi, pi, d, d, i, pd, pd, pd, pd]
        L.orc_matvec.argtypes = [ctypes.c_char_p, i, i, pi, pi, pi, pd, pd, c, pd, i, c, pd,
                                 d, pd, pd]
        L.orc_dot.argtypes = [i, pd, pd]
        L.orc_dot.restype = d
        L.orc_dot_blocked.argtypes = [i, pd, pd, i, i]
        L.orc_dot_blocked.restype = d
        L.orc_precd1.argtypes = [i, i, pi, pi, pi, i, pd, pd, P(c), pd, i, c, pd, pd]
        L.orc_solve.argtypes = [i, i, pi, pi, pi, pd, pd, pd, P(c), pd, i, c, i, i, i, d, i, i,
                                i, pi, pd, pi, i]
        L.orc_set_threads.argtypes = [i]
        L.orc_solve_mixed.argtypes = [i, i, pi, pi, pi, pd, pd, pd, c, pd, c, i, d, d, i, i, i,
                                      i, pi, pi, pd]
        _lib = L
    return _lib


def set_threads(n):
    """Host threads of the restatement's large-case runs (1: the sequential
    code).  Loops with independent iterations are shared out; every sum
    keeps its order, so the results are the same bits with any count."""
    lib().orc_set_threads(int(n))


class threads:
    """Context manager: run the enclosed oracle calls on n host threads
    (all of the host's by default), then return to one."""

    def __init__(self, n=None):
        self.n = n or (os.cpu_count() or 1)

    def __enter__(self):
        set_threads(self.n)
        return self

    def __exit__(self, *exc):
        set_threads(1)


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _pi(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _cols(ikle0):
    """0-based IKLE (nelem, 3) -> three contiguous int32 columns."""
    ik = np.ascontiguousarray(np.asarray(ikle0, dtype=np.int32).T)
    return ik, ik[0], ik[1], ik[2]


def wave_matrix(x, y, ikle0, coef):
    """A = M + coef_e K_e as PROPAG builds AM1 (mass MT01AA + P0 diffusion
    MT02AA, diagonals by ASSVEC).  Returns dm (npoin,), xm (3, nelem)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    coef = np.ascontiguousarray(coef, dtype=np.float64)
    ik, a, b, c = _cols(ikle0)
    n, ne = x.size, ik.shape[1]
    dm = np.empty(n)
    xm = np.empty((3, ne))
    st = lib().orc_wave_matrix(n, ne, _pd(x), _pd(y), _pi(a), _pi(b), _pi(c), _pd(coef),
                               _pd(dm), _pd(xm))
    if st:
        raise ValueError("orc_wave_matrix status %d" % st)
    return dm, xm


def mass_diff_matrix(x, y, ikle0, u, v=None, kind=11, xmul_mass=1.0, xmul_dif=1.0):
    """AM1 = MT01AA(xmul_mass) + MT02AA(xmul_dif) as PROPAG assembles it:
    kind 10 MATDIF with u per element, 11 MATDIF with u per node, 12
    MATDIFUV with u and v per node.  Returns dm (npoin,), xm (3, nelem)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
    ik, a, b, c = _cols(ikle0)
    n, ne = x.size, ik.shape[1]
    dm = np.empty(n)
    xm = np.empty((3, ne))
    st = lib().orc_mass_diff_matrix(n, ne, _pd(x), _pd(y), _pi(a), _pi(b), _pi(c),
                                    float(xmul_mass), float(xmul_dif), int(kind), _pd(u),
                                    None if vv is None else _pd(vv), _pd(dm), _pd(xm))
    if st:
        raise ValueError("orc_mass_diff_matrix status %d" % st)
    return dm, xm


def unit_stiffness(x, y, ikle0):
    """Off-diagonal terms (3, nelem) of the unit-coefficient MT02AA matrix."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    ik, a, b, c = _cols(ikle0)
    kxm = np.empty((3, ik.shape[1]))
    st = lib().orc_wave_matrix_parts(x.size, ik.shape[1], _pd(x), _pd(y), _pi(a), _pi(b),
                                     _pi(c), _pd(kxm))
    if st:
        raise ValueError("orc_wave_matrix_parts status %d" % st)
    return kxm


def matvec(op, ikle0, dm, typdia, xm, typext, y, c=0.0, x=None):
    """MATVEC(OP,X,A,Y,C): returns the new X (a copy)."""
    ik, a, b, cc = _cols(ikle0)
    n, ne = np.asarray(y).size, ik.shape[1]
    xm = np.ascontiguousarray(xm, dtype=np.float64).reshape(-1, ne)
    out = np.zeros(n) if x is None else np.array(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    t = np.empty(n)
    w = np.empty(3 * ne + 1)
    st = lib().orc_matvec(op.encode(), n, ne, _pi(a), _pi(b), _pi(cc), _pd(out), _pd(dm),
                          typdia.encode(), _pd(xm), ne, typext.encode(), _pd(y), c, _pd(t), _pd(w))
    if st:
        raise ValueError("orc_matvec status %d" % st)
    return out


def dot(x, y, mode=DOT_SEQUENTIAL, nblocks=1, nthreads=256):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    L = lib()
    if mode == DOT_BLOCKED:
        return L.orc_dot_blocked(x.size, _pd(x), _pd(y), nblocks, nthreads)
    if mode in (DOT_COMP_SEQUENTIAL, DOT_COMP_BLOCKED):
        P = ctypes.POINTER
        L.orc_dot_comp.argtypes = [ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double)]
        L.orc_dot_comp.restype = ctypes.c_double
        L.orc_dot_blocked_comp.argtypes = [ctypes.c_int, P(ctypes.c_double),
                                           P(ctypes.c_double), ctypes.c_int, ctypes.c_int]
        L.orc_dot_blocked_comp.restype = ctypes.c_double
        if mode == DOT_COMP_SEQUENTIAL:
            return L.orc_dot_comp(x.size, _pd(x), _pd(y))
        return L.orc_dot_blocked_comp(x.size, _pd(x), _pd(y), nblocks, nthreads)
    return L.orc_dot(x.size, _pd(x), _pd(y))


def solve(ikle0, dm, typdia, xm, typext, b, x0=None, precon=2, nitmax=100000, eps=1e-8,
          slv=1, dot_mode=DOT_SEQUENTIAL, nblocks=1, nthreads=256, krylov=3):
    """SOLVE(X,A,B) with SLV=1.  Works on copies; returns a dict with x, the
    mutated b/dm/xm/typdia (as the reference leaves them), status, nit,
    relres, relat."""
    ik, a, bb, c = _cols(ikle0)
    n, ne = np.asarray(b).size, ik.shape[1]
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.array(b, dtype=np.float64)
    dm = np.array(dm, dtype=np.float64)
    xm = np.array(xm, dtype=np.float64).reshape(-1, ne).copy()
    td = ctypes.c_char(typdia.encode())
    nit, relat = ctypes.c_int(0), ctypes.c_int(0)
    relres = ctypes.c_double(0.0)
    st = lib().orc_solve(n, ne, _pi(a), _pi(bb), _pi(c), _pd(x), _pd(b), _pd(dm),
                         ctypes.byref(td), _pd(xm), ne, typext.encode(), slv, precon, nitmax,
                         eps, dot_mode, nblocks, nthreads, ctypes.byref(nit),
                         ctypes.byref(relres), ctypes.byref(relat), krylov)
    return dict(x=x, b=b, dm=dm, xm=xm, typdia=td.value.decode(), status=st, nit=nit.value,
                relres=relres.value, relat=relat.value)


def solve_mixed(ikle0, dm, typdia, xm, b, x0=None, precon=2, inner_tol=0.1, outer_tol=1e-8,
                max_outer=50, max_inner=100000, nblocks=1, nthreads=256):
    """Mixed-precision solve (binary32 inner CG, binary64 refinement) in the
    device kernels' exact operation order."""
    ik, a, bb, c = _cols(ikle0)
    n, ne = np.asarray(b).size, ik.shape[1]
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    xm = np.ascontiguousarray(xm, dtype=np.float64).reshape(3, ne)
    outer, inner = ctypes.c_int(0), ctypes.c_int(0)
    relres = ctypes.c_double(0.0)
    st = lib().orc_solve_mixed(n, ne, _pi(a), _pi(bb), _pi(c), _pd(x), _pd(b), _pd(dm),
                               typdia.encode(), _pd(xm), b"S", precon, inner_tol, outer_tol,
                               max_outer, max_inner, nblocks, nthreads, ctypes.byref(outer),
                               ctypes.byref(inner), ctypes.byref(relres))
    return dict(x=x, status=st, outer=outer.value, inner=inner.value, relres=relres.value)


def dot_batch(x, y, nthreads=1024, npt=1):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    L = lib()
    L.orc_dot_batch.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int]
    L.orc_dot_batch.restype = ctypes.c_double
    return L.orc_dot_batch(x.size, _pd(x), _pd(y), nthreads, npt)


def solve_mixed_batch(ikle0, dm, typdia, xm, b, x0=None, precon=2, inner_tol=0.1,
                      outer_tol=1e-8, max_outer=1000, max_inner=1000000, nthreads=1024, npt=1):
    """One instance of the batched mixed-precision solver, in the batched
    kernel's dot order (tiles of nthreads*npt nodes, warp sum of tiles)."""
    ik, a, bb, c = _cols(ikle0)
    n, ne = np.asarray(b).size, ik.shape[1]
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    xm = np.ascontiguousarray(xm, dtype=np.float64).reshape(3, ne)
    L = lib()
    P = ctypes.POINTER
    d, i, ch = ctypes.c_double, ctypes.c_int, ctypes.c_char
    L.orc_solve_mixed_batch.argtypes = [i, i, P(i), P(i), P(i), P(d), P(d), P(d), ch, P(d), ch,
                                        i, d, d, i, i, i, i, P(i), P(i), P(d)]
    outer, inner = ctypes.c_int(0), ctypes.c_int(0)
    relres = ctypes.c_double(0.0)
    st = L.orc_solve_mixed_batch(n, ne, _pi(a), _pi(bb), _pi(c), _pd(x), _pd(b), _pd(dm),
                                 typdia.encode(), _pd(xm), b"S", precon, inner_tol, outer_tol,
                                 max_outer, max_inner, nthreads, npt, ctypes.byref(outer),
                                 ctypes.byref(inner), ctypes.byref(relres))
    return dict(x=x, status=st, outer=outer.value, inner=inner.value, relres=relres.value)


def solve_mixed_batch_seg(g1, g2, dm, typdia, xa, b, x0=None, precon=2, inner_tol=0.1,
                          outer_tol=1e-8, max_outer=1000, max_inner=1000000, nthreads=1024,
                          npt=1):
    """One instance of the batched mixed-precision solver on a segment-storage
    matrix (symmetric XA(NSEG)), in the batched kernel's dot order."""
    g1, g2 = _i32(g1), _i32(g2)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = b.size
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    xa = np.ascontiguousarray(xa, dtype=np.float64).ravel()
    L = lib()
    P = ctypes.POINTER
    d, i, ch = ctypes.c_double, ctypes.c_int, ctypes.c_char
    L.orc_solve_mixed_batch_seg.argtypes = [i, i, P(i), P(i), P(d), P(d), P(d), ch, P(d), ch, i,
                                            d, d, i, i, i, i, P(i), P(i), P(d)]
    outer, inner = ctypes.c_int(0), ctypes.c_int(0)
    relres = ctypes.c_double(0.0)
    st = L.orc_solve_mixed_batch_seg(n, g1.size, _pi(g1), _pi(g2), _pd(x), _pd(b), _pd(dm),
                                     typdia.encode(), _pd(xa), b"S", precon, inner_tol,
                                     outer_tol, max_outer, max_inner, nthreads, npt,
                                     ctypes.byref(outer), ctypes.byref(inner),
                                     ctypes.byref(relres))
    return dict(x=x, status=st, outer=outer.value, inner=inner.value, relres=relres.value)


def solve_omp(ikle0, dm, xm, b, x0=None, nitmax=1000000, eps=1e-8, nthreads=None):
    """Binary64 SOLVE (PRECON 2, symmetric) on `nthreads` host threads."""
    ik, a, bb, c = _cols(ikle0)
    n, ne = np.asarray(b).size, ik.shape[1]
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    xm = np.ascontiguousarray(xm, dtype=np.float64).reshape(3, ne)
    L = lib()
    P = ctypes.POINTER
    d, i = ctypes.c_double, ctypes.c_int
    L.orc_solve_omp.argtypes = [i, i, P(i), P(i), P(i), P(d), P(d), P(d), P(d), i, d, i, P(i),
                                P(d)]
    nit, relres = ctypes.c_int(0), ctypes.c_double(0.0)
    st = L.orc_solve_omp(n, ne, _pi(a), _pi(bb), _pi(c), _pd(x), _pd(b), _pd(dm), _pd(xm),
                         nitmax, eps, nthreads or (os.cpu_count() or 1), ctypes.byref(nit),
                         ctypes.byref(relres))
    return dict(x=x, status=st, nit=nit.value, relres=relres.value)


# -- segment storage (STO=3) ------------------------------------------------

def _seg_lib():
    L = lib()
    if not getattr(L, "_seg_ready", False):
        P = ctypes.POINTER
        d, i, c = ctypes.c_double, ctypes.c_int, ctypes.c_char
        pd, pi = P(d), P(i)
        L.orc_stoseg.argtypes = [i, i, pi, pi, pi, i, pi, pi, pi, pi, pi, pi, pi]
        L.orc_assex3.argtypes = [i, pi, pi, c, pd, i, i, pd]
        L.orc_mvseg.argtypes = [ctypes.c_char_p, i, i, pi, pi, pd, pd, c, pd, c, pd, d]
        L.orc_solve_seg.argtypes = [i, i, pi, pi, pd, pd, pd, P(c), pd, c, i, i, i, d, i, i, i,
                                    pi, pd, pi, i]
        L.orc_solve_mixed_seg.argtypes = [i, i, pi, pi, pd, pd, pd, c, pd, c, i, d, d, i, i, i,
                                          i, pi, pi, pd]
        L._seg_ready = True
    return L


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def stoseg(ikle0, npoin, nelbor, nulone):
    """STOSEG numbering: boundary segments first (element nelbor[s], face
    nulone[s], in that order), then the remaining element faces.  Returns
    g1, g2 (0-based GLOSEG columns), eltseg and oriseg (3, nelem)."""
    ik, a, b, c = _cols(ikle0)
    ne = ik.shape[1]
    nelbor, nulone = _i32(nelbor), _i32(nulone)
    cap = 3 * ne + 1
    g1, g2 = np.empty(cap, np.int32), np.empty(cap, np.int32)
    es, ori = np.empty((3, ne), np.int32), np.empty((3, ne), np.int32)
    nseg = ctypes.c_int(0)
    st = _seg_lib().orc_stoseg(npoin, ne, _pi(a), _pi(b), _pi(c), nelbor.size, _pi(nelbor),
                               _pi(nulone), _pi(g1), _pi(g2), _pi(es), _pi(ori),
                               ctypes.byref(nseg))
    if st:
        raise ValueError("orc_stoseg status %d" % st)
    n = nseg.value
    return g1[:n].copy(), g2[:n].copy(), es, ori


def assex3(eltseg, oriseg, typext, xmt, nseg):
    """EBE off-diagonal terms (3|6, nelem) -> segment XA: (nseg,) for 'S',
    (2, nseg) for 'Q'."""
    es, ori = _i32(eltseg), _i32(oriseg)
    ne = es.shape[1]
    xmt = np.ascontiguousarray(xmt, dtype=np.float64).reshape(-1, ne)
    xa = np.empty((1 if typext == "S" else 2) * nseg)
    st = _seg_lib().orc_assex3(ne, _pi(es), _pi(ori), typext.encode(), _pd(xmt), ne, nseg,
                               _pd(xa))
    if st:
        raise ValueError("orc_assex3 status %d" % st)
    return xa if typext == "S" else xa.reshape(2, nseg)


def mvseg(op, g1, g2, dm, typdia, xa, typext, y, c=0.0, x=None):
    """MATVEC on segment storage (MVSEG): returns the new X (a copy)."""
    g1, g2 = _i32(g1), _i32(g2)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = y.size
    out = np.zeros(n) if x is None else np.array(x, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    xa = np.ascontiguousarray(xa, dtype=np.float64).ravel()
    st = _seg_lib().orc_mvseg(op.encode(), n, g1.size, _pi(g1), _pi(g2), _pd(out), _pd(dm),
                              typdia.encode(), _pd(xa), typext.encode(), _pd(y), c)
    if st:
        raise ValueError("orc_mvseg status %d" % st)
    return out


def solve_seg(g1, g2, dm, typdia, xa, typext, b, x0=None, precon=2, nitmax=100000, eps=1e-8,
              slv=1, dot_mode=DOT_SEQUENTIAL, nblocks=1, nthreads=256, krylov=3):
    """SOLVE(SLV=1) on a segment-storage matrix; same outputs as solve()
    (with 'xa' for the mutated off-diagonal terms)."""
    g1, g2 = _i32(g1), _i32(g2)
    b = np.array(b, dtype=np.float64)
    n = b.size
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    dm = np.array(dm, dtype=np.float64)
    xa = np.array(xa, dtype=np.float64).ravel().copy()
    td = ctypes.c_char(typdia.encode())
    nit, relat = ctypes.c_int(0), ctypes.c_int(0)
    relres = ctypes.c_double(0.0)
    st = _seg_lib().orc_solve_seg(n, g1.size, _pi(g1), _pi(g2), _pd(x), _pd(b), _pd(dm),
                                  ctypes.byref(td), _pd(xa), typext.encode(), slv, precon,
                                  nitmax, eps, dot_mode, nblocks, nthreads, ctypes.byref(nit),
                                  ctypes.byref(relres), ctypes.byref(relat), krylov)
    return dict(x=x, b=b, dm=dm, xa=xa, typdia=td.value.decode(), status=st, nit=nit.value,
                relres=relres.value, relat=relat.value)


def solve_mixed_seg(g1, g2, dm, typdia, xa, b, x0=None, precon=2, inner_tol=0.1,
                    outer_tol=1e-8, max_outer=1000, max_inner=1000000, nblocks=1, nthreads=256):
    """Mixed-precision solve on a symmetric segment-storage matrix in the
    device kernels' exact operation order."""
    g1, g2 = _i32(g1), _i32(g2)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = b.size
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    xa = np.ascontiguousarray(xa, dtype=np.float64).ravel()
    outer, inner = ctypes.c_int(0), ctypes.c_int(0)
    relres = ctypes.c_double(0.0)
    st = _seg_lib().orc_solve_mixed_seg(n, g1.size, _pi(g1), _pi(g2), _pd(x), _pd(b), _pd(dm),
                                        typdia.encode(), _pd(xa), b"S", precon, inner_tol,
                                        outer_tol, max_outer, max_inner, nblocks, nthreads,
                                        ctypes.byref(outer), ctypes.byref(inner),
                                        ctypes.byref(relres))
    return dict(x=x, status=st, outer=outer.value, inner=inner.value, relres=relres.value)


def diri01(ikle0, dm, typdia, xm, typext, nbor0, limdir, kdir, fbor, sm, f, maskpt=None):
    """DIRI01 with boundary values (nbor0 0-based).  Returns (xm, sm, f) as
    modified (copies)."""
    L = lib()
    if not getattr(L, "_diri_ready", False):
        P = ctypes.POINTER
        d, i, c = ctypes.c_double, ctypes.c_int, ctypes.c_char
        pd, pi = P(d), P(i)
        L.orc_diri01.argtypes = [i, i, pi, pi, pi, pd, c, pd, c, i, pi, pi, i, pd, pd, pd,
                                 ctypes.c_void_p]
        L.orc_diri01_seg.argtypes = [i, i, pi, pi, pd, c, pd, c, i, pi, pi, i, pd, pd, pd,
                                     ctypes.c_void_p]
        L._diri_ready = True
    ik, a, b, c = _cols(ikle0)
    ne = ik.shape[1]
    xm = np.array(xm, dtype=np.float64).reshape(-1, ne).copy()
    sm, f = np.array(sm, dtype=np.float64), np.array(f, dtype=np.float64)
    nb, ld = _i32(nbor0), _i32(limdir)
    fb = np.ascontiguousarray(fbor, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    mk = None if maskpt is None else np.ascontiguousarray(maskpt, dtype=np.float64)
    st = L.orc_diri01(sm.size, ne, _pi(a), _pi(b), _pi(c), _pd(dm), typdia.encode(), _pd(xm),
                      typext.encode(), nb.size, _pi(nb), _pi(ld), kdir, _pd(fb), _pd(sm), _pd(f),
                      None if mk is None else mk.ctypes.data_as(ctypes.c_void_p))
    if st:
        raise ValueError("orc_diri01 status %d" % st)
    return xm, sm, f


def diri01_seg(g1, g2, dm, typdia, xa, typext, nbor0, limdir, kdir, fbor, sm, f, maskpt=None):
    """DIRI01 on a segment-storage matrix.  Returns (xa, sm, f) (copies)."""
    L = lib()
    if not getattr(L, "_diri_ready", False):
        diri01(np.zeros((1, 3), np.int32), np.ones(3), "Q", np.zeros((3, 1)), "S",
               np.zeros(0, np.int32), np.zeros(0, np.int32), 1, np.zeros(0), np.zeros(3),
               np.zeros(3))
    g1, g2 = _i32(g1), _i32(g2)
    xa = np.array(xa, dtype=np.float64).ravel().copy()
    sm, f = np.array(sm, dtype=np.float64), np.array(f, dtype=np.float64)
    nb, ld = _i32(nbor0), _i32(limdir)
    fb = np.ascontiguousarray(fbor, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    mk = None if maskpt is None else np.ascontiguousarray(maskpt, dtype=np.float64)
    st = L.orc_diri01_seg(sm.size, g1.size, _pi(g1), _pi(g2), _pd(dm), typdia.encode(), _pd(xa),
                          typext.encode(), nb.size, _pi(nb), _pi(ld), kdir, _pd(fb), _pd(sm),
                          _pd(f), None if mk is None else mk.ctypes.data_as(ctypes.c_void_p))
    if st:
        raise ValueError("orc_diri01_seg status %d" % st)
    return xa, sm, f
