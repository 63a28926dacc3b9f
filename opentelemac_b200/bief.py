"""Host-side mirror of BIEF's SOLVE / MATVEC interface over libbief_b200.

    SOLVE(X,A,B,TB,CFG,INFOGR,MESH,AUX)   sources/utils/bief/solve.f:2-5
    MATVEC(OP,X,A,Y,C,MESH,LEGO)          sources/utils/bief/matvec.f:2-5

`Mesh` stands for the IKLE/NPOIN/NELEM part of BIEF_MESH, `Matrix` for a
BIEF_OBJ matrix with EBE storage (STO=1) and `SlvCfg` for SLVCFG.  Vectors
are numpy float64 arrays (host path: the library copies them to the device
and back) or torch CUDA float64 tensors (device path, no copies).

Errors: the reference aborts with PLANTE(1); here a negative status raises
BiefError.  A solve that stops at NITMAX returns normally with cfg.ok = 0
(the reference only prints a message in that case).
"""
import ctypes

import numpy as np

from . import _native
from ._native import BiefError, SlvCfg  # noqa: F401  (re-exported)


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if _is_torch(a):
        if not a.is_cuda or not a.is_contiguous():
            raise ValueError("torch tensors must be contiguous CUDA tensors")
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def _dev(a, n, mesh, what, dtype="float64"):
    """Pointer to a torch tensor handed to a device entry point, after the
    checks the library cannot make on a device address: contiguous, on the
    mesh's GPU, of the expected dtype, exactly n values."""
    import torch
    if not _is_torch(a) or not a.is_cuda or not a.is_contiguous():
        raise ValueError(f"{what}: a contiguous CUDA tensor is expected")
    if a.dtype != getattr(torch, dtype):
        raise TypeError(f"{what}: {dtype} expected, got {a.dtype}")
    if a.device.index != mesh.device:
        raise ValueError(f"{what}: tensor on cuda:{a.device.index}, mesh on cuda:{mesh.device}")
    if a.numel() != n:
        raise ValueError(f"{what}: {a.numel()} values, {n} expected")
    return ctypes.c_void_p(a.data_ptr())


def _host_in(a, n, what):
    """A host input array as the library reads it: float64, contiguous,
    exactly n values."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != n:
        raise ValueError(f"{what}: {a.size} values, {n} expected")
    return a


def _stream(a):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)


def _check(st, what):
    if st < 0:
        raise BiefError(st, what)
    return st


class Mesh:
    """Mesh connectivity on one GPU (owns the native handle).

    ikle0: (nelem, 3) 0-based node numbers of each triangle, or use
    Mesh.from_fortran for the reference's IKLE(NELMAX,3) 1-based layout."""

    def __init__(self, ikle0, npoin, device=0):
        ik = np.asarray(ikle0)
        if ik.ndim != 2 or ik.shape[1] != 3:
            raise ValueError("ikle0 must have shape (nelem, 3)")
        nelem = ik.shape[0]
        fort = np.ascontiguousarray((ik.T + 1).astype(np.int32)).ravel()
        self._init(fort, npoin, nelem, nelem, device)

    @classmethod
    def from_fortran(cls, ikle, npoin, nelem, nelmax, device=0):
        self = cls.__new__(cls)
        self._init(np.ascontiguousarray(ikle, dtype=np.int32).ravel(), npoin, nelem, nelmax,
                   device)
        return self

    def _init(self, fort, npoin, nelem, nelmax, device):
        self.npoin, self.nelem, self.nelmax, self.device = int(npoin), int(nelem), int(nelmax), device
        self._h = ctypes.c_void_p()
        L = _native.lib()
        _check(L.bief_mesh_create(self.npoin, self.nelem, self.nelmax,
                                  fort.ctypes.data_as(ctypes.c_void_p), device,
                                  ctypes.byref(self._h)), "bief_mesh_create")

    @property
    def handle(self):
        return self._h

    def launch_info(self):
        """(blocks, threads) of the persistent solver: the dot-product tree."""
        g, t = ctypes.c_int(), ctypes.c_int()
        _native.lib().bief_launch_info(self._h, ctypes.byref(g), ctypes.byref(t))
        return g.value, t.value

    def set_blocks_per_sm(self, n=0):
        """Residency of the persistent solvers: 1 or 2 blocks per SM, 0 for
        the automatic choice (2 when the binary32 working set, about 80 B per
        node, exceeds 2.25 times the L2: about 3.5M nodes on a B200).
        Sets the dot-product tree's shape (launch_info)."""
        _check(_native.lib().bief_set_blocks_per_sm(self._h, int(n)), "bief_set_blocks_per_sm")

    MATVEC_FORMATS = ("ikle", "local", "band", "any")

    def matvec_format(self):
        """Gather records of the standalone MATVEC for this mesh: 'local' (6 B
        per entry), 'band' (8 B), 'any' (12 B) or 'ikle' (a node in more than
        255 elements: element index, then IKLE)."""
        f = ctypes.c_int()
        _check(_native.lib().bief_matvec_format(self._h, ctypes.byref(f)), "bief_matvec_format")
        return self.MATVEC_FORMATS[f.value]

    def last_timing(self):
        s, m = ctypes.c_float(), ctypes.c_float()
        _native.lib().bief_last_timing(self._h, ctypes.byref(s), ctypes.byref(m))
        return s.value, m.value

    def kernel_launches(self):
        return int(_native.lib().bief_kernel_launches(self._h))

    def set_segments(self, g1, g2):
        """Segment numbering (MESH%GLOSEG) from 0-based end points g1, g2
        (see meshgen.segments for the STOSEG conventions).  Enables segment
        storage (STO=3) matrices on this mesh."""
        g1 = np.asarray(g1)
        g2 = np.asarray(g2)
        gl = np.ascontiguousarray(np.concatenate([g1, g2]).astype(np.int32) + 1)
        nseg = int(g1.size)
        _check(_native.lib().bief_set_segments(self._h, nseg, nseg,
                                               gl.ctypes.data_as(ctypes.c_void_p)),
               "bief_set_segments")
        self.nseg = nseg
        return self

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _native.lib().bief_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Matrix:
    """EBE matrix A (A%D, A%X, TYPDIA, TYPEXT) stored on the mesh's handle.

    dm: (npoin,) diagonal; xm: (ndiag, nelem) off-diagonal terms, columns
    M12, M13, M23 (+ M21, M31, M32 for typext 'Q').  The handle holds one
    matrix: creating a second Matrix on the same Mesh replaces the first."""

    def __init__(self, mesh, dm=None, xm=None, typdia="Q", typext="S"):
        self.mesh = mesh
        self.typdia, self.typext = typdia, typext
        if dm is not None:
            self.set(dm, xm, typdia, typext)

    def set(self, dm, xm, typdia="Q", typext="S"):
        L = _native.lib()
        if _is_torch(dm):
            m = self.mesh
            nd = {"S": 3, "Q": 6, "0": 0}.get(typext, 0)
            pxm = _dev(xm, nd * m.nelem, m, "xm") if nd else None
            _check(L.bief_set_matrix_dev(m.handle, _dev(dm, m.npoin, m, "dm"), pxm,
                                         typdia.encode(), typext.encode()), "bief_set_matrix_dev")
        else:
            dm = np.ascontiguousarray(dm, dtype=np.float64)
            nd = {"S": 3, "Q": 6, "0": 0}[typext]
            if dm.size != self.mesh.npoin:
                raise ValueError("dm must have npoin = %d values" % self.mesh.npoin)
            xm = self._host_xm(xm, nd) if nd else np.zeros(1)
            _check(L.bief_set_matrix(self.mesh.handle, _ptr(dm), _ptr(xm), typdia.encode(),
                                     typext.encode()), "bief_set_matrix")
        self.typdia, self.typext = typdia, typext
        return self

    def _host_xm(self, xm, nd):
        """XM as the host entry points read it, XM(NELMAX,NDIAG): (nd, nelem)
        input is padded to the mesh's NELMAX; (nd, nelmax) is taken as is."""
        xm = np.asarray(xm, dtype=np.float64)
        ne, nmax = self.mesh.nelem, self.mesh.nelmax
        if xm.size == nd * nmax:
            return np.ascontiguousarray(xm.reshape(nd, nmax))
        if xm.size == nd * ne:
            out = np.zeros((nd, nmax))
            out[:, :ne] = xm.reshape(nd, ne)
            return out
        raise ValueError("xm must have %d x nelem (%d) or %d x nelmax (%d) values"
                         % (nd, ne, nd, nmax))

    def get(self):
        """Stored (dm, xm, typdia) as numpy arrays: xm (ndiag, nelem) for EBE
        storage, (ncol, nseg) for segment storage."""
        seg = self.storage == 3
        nd = ({"S": 1, "Q": 2, "0": 0} if seg else {"S": 3, "Q": 6, "0": 0})[self.typext]
        dm = np.empty(self.mesh.npoin)
        # the host entry point writes EBE columns with the NELMAX pitch
        xm = np.empty((max(nd, 1), self.mesh.nseg if seg else self.mesh.nelmax))
        td = ctypes.create_string_buffer(2)
        _check(_native.lib().bief_get_matrix(self.mesh.handle, _ptr(dm), _ptr(xm), td),
               "bief_get_matrix")
        self.typdia = td.value.decode()
        return dm, (xm[:nd] if seg else xm[:nd, :self.mesh.nelem]), self.typdia

    def get_dev(self):
        """Stored (dm, xm) as torch CUDA float64 tensors on the mesh's device,
        shaped as get() returns them (TYPDIA is get()'s)."""
        import torch
        seg = self.storage == 3
        nd = ({"S": 1, "Q": 2, "0": 0} if seg else {"S": 3, "Q": 6, "0": 0})[self.typext]
        dev = torch.device("cuda", self.mesh.device)
        dm = torch.empty(self.mesh.npoin, dtype=torch.float64, device=dev)
        xm = torch.empty((max(nd, 1), self.mesh.nseg if seg else self.mesh.nelem),
                         dtype=torch.float64, device=dev)
        _check(_native.lib().bief_get_matrix_dev(self.mesh.handle, _ptr(dm), _ptr(xm),
                                                 _stream(dm)), "bief_get_matrix_dev")
        torch.cuda.current_stream(dev).synchronize()
        return dm, xm[:nd]

    def set_seg(self, da, xa, typdia="Q", typext="S"):
        """Segment storage (STO=3): DA (npoin,) and XA (nseg,) for 'S' or
        (2, nseg) for 'Q'; numpy arrays or torch CUDA tensors."""
        L = _native.lib()
        m = self.mesh
        nc = {"S": 1, "Q": 2, "0": 0}.get(typext, 0)
        if getattr(m, "nseg", None) is None:      # as the library answers
            raise BiefError(_native.BIEF_ERR_NO_MATRIX, "segment matrix without numbering")
        if _is_torch(da):
            pxa = _dev(xa, nc * m.nseg, m, "xa") if nc else None
            _check(L.bief_set_matrix_seg_dev(m.handle, _dev(da, m.npoin, m, "da"), pxa,
                                             typdia.encode(), typext.encode()),
                   "bief_set_matrix_seg_dev")
        else:
            da = _host_in(da, m.npoin, "da")
            xa = _host_in(np.asarray(xa).ravel(), nc * m.nseg, "xa") if nc else np.zeros(1)
            _check(L.bief_set_matrix_seg(self.mesh.handle, _ptr(da), _ptr(xa), typdia.encode(),
                                         typext.encode()), "bief_set_matrix_seg")
        self.typdia, self.typext = typdia, typext
        return self

    def to_segments(self):
        """ASSEX3: the stored EBE matrix becomes segment storage."""
        _check(_native.lib().bief_ebe_to_seg(self.mesh.handle, None), "bief_ebe_to_seg")
        return self

    @property
    def storage(self):
        """1 (EBE) or 3 (segments)."""
        return _check(_native.lib().bief_matrix_storage(self.mesh.handle), "bief_matrix_storage")

    def assemble_wave(self, xc, yc, coef):
        """A = M + coef_e K_e from device coordinates and coefficients
        (torch CUDA float64 tensors)."""
        m = self.mesh
        _check(_native.lib().bief_assemble_wave_dev(
            m.handle, _dev(xc, m.npoin, m, "x"), _dev(yc, m.npoin, m, "y"),
            _dev(coef, m.nelem, m, "coef"), _stream(xc)), "bief_assemble_wave_dev")
        self.typdia, self.typext = "Q", "S"
        return self

    def assemble_mass_diff(self, xc, yc, u, v=None, kind=11, xmul_mass=1.0, xmul_dif=1.0):
        """AM1 = MT01AA(xmul_mass) + MT02AA(xmul_dif) as PROPAG builds it:
        kind 10 MATDIF with u per element, 11 MATDIF with u per node, 12
        MATDIFUV with u and v per node (PROPAG: u = DM1, v = HPROP,
        xmul_dif = -1).  torch CUDA float64 tensors."""
        if kind == 12 and v is None:
            raise ValueError("MATDIFUV needs v")
        m = self.mesh
        nu = m.nelem if kind == 10 else m.npoin
        _check(_native.lib().bief_assemble_mass_diff_dev(
            m.handle, _dev(xc, m.npoin, m, "x"), _dev(yc, m.npoin, m, "y"), float(xmul_mass),
            float(xmul_dif), int(kind), _dev(u, nu, m, "u"),
            None if v is None else _dev(v, m.npoin, m, "v"), _stream(xc)),
            "bief_assemble_mass_diff_dev")
        self.typdia, self.typext = "Q", "S"
        return self


def solve(x, A, b, cfg, infogr=False, mutate=False, modass=1):
    """SOLVE(X,A,B,...,CFG,INFOGR,...) for CFG.slv = 1 (GRACJG), 2 (RESCJG),
    3 (EQUNOR), 4 (ERRMIN), 5 (CGSQUA), 6 (CGSTAB) or 7 (GMRES).

    x holds the initial guess and receives the solution.  With mutate=True
    the reference's side effects are reproduced: b becomes D.b and A is
    replaced by D.A.D (TYPDIA 'I').  modass=3 selects compensated dot
    products (every method).  Returns (status, nit, relres)."""
    L = _native.lib()
    flags = (_native.BIEF_SOLVE_MUTATE_INPUTS if mutate else 0) | (
        _native.BIEF_SOLVE_INFOGR if infogr else 0) | (
        _native.BIEF_SOLVE_MODASS3 if modass == 3 else 0)
    relres = ctypes.c_double()
    m = A.mesh
    if _is_torch(x):
        st = L.bief_solve_dev(m.handle, _dev(x, m.npoin, m, "x"), _dev(b, m.npoin, m, "b"),
                              ctypes.byref(cfg), flags, ctypes.byref(relres), _stream(x))
    else:
        _host_vec(x, A.mesh.npoin)
        _host_vec(b, A.mesh.npoin)
        st = L.bief_solve(A.mesh.handle, _ptr(x), _ptr(b), ctypes.byref(cfg), flags,
                          ctypes.byref(relres))
    _check(st, "SOLVE")
    if mutate:
        A.typdia = A.get()[2] if not _is_torch(x) else A.typdia
    return st, cfg.nit, relres.value


def solve_mixed(x, A, b, precon=2, inner_tol=0.1, outer_tol=1e-8, max_outer=1000,
                max_inner=1000000):
    """Mixed-precision solve (binary32 inner CG, binary64 refinement each
    time the binary32 residual has dropped by inner_tol).
    Returns (status, outer_steps, inner_iterations, relres)."""
    L = _native.lib()
    o, i = ctypes.c_int(), ctypes.c_int()
    relres = ctypes.c_double()
    m = A.mesh
    if _is_torch(x):
        st = L.bief_solve_mixed_dev(m.handle, _dev(x, m.npoin, m, "x"), _dev(b, m.npoin, m, "b"),
                                    precon, inner_tol, outer_tol, max_outer, max_inner,
                                    ctypes.byref(o), ctypes.byref(i), ctypes.byref(relres),
                                    _stream(x))
    else:
        _host_vec(x, A.mesh.npoin)
        b = _host_in(b, A.mesh.npoin, "b")
        st = L.bief_solve_mixed(A.mesh.handle, _ptr(x), _ptr(b), precon, inner_tol, outer_tol,
                                max_outer, max_inner, ctypes.byref(o), ctypes.byref(i),
                                ctypes.byref(relres))
    _check(st, "SOLVE (mixed)")
    return st, o.value, i.value, relres.value


def matvec(op, x, A, y, c=0.0):
    """MATVEC(OP,X,A,Y,C,MESH,LEGO=.TRUE.): X updated in place."""
    L = _native.lib()
    opb = op.encode() if isinstance(op, str) else op
    m = A.mesh
    if _is_torch(x):
        st = L.bief_matvec_dev(m.handle, opb, _dev(x, m.npoin, m, "x"),
                               _dev(y, m.npoin, m, "y"), float(c), _stream(x))
    else:
        _host_vec(x, A.mesh.npoin)
        y = _host_in(y, A.mesh.npoin, "y")
        st = L.bief_matvec(A.mesh.handle, opb, _ptr(x), _ptr(y), float(c))
    _check(st, "MATVEC")
    return x


def matvec32(x, A, y):
    """X = A Y in binary32 on the binary32 copy of A that the mixed-precision
    inner CG uses (symmetric matrices); x and y are float32 CUDA tensors,
    x updated in place.  No reference counterpart."""
    m = A.mesh
    if not (_is_torch(x) and _is_torch(y)):
        raise TypeError("matvec32 takes float32 CUDA tensors")
    st = _native.lib().bief_matvec32_dev(m.handle, _dev(x, m.npoin, m, "x", "float32"),
                                         _dev(y, m.npoin, m, "y", "float32"), _stream(x))
    _check(st, "MATVEC32")
    return x


def diri01(A, nbor, limdir, kdir, fbor, sm, f, maskpt=None):
    """DIRI01 for Dirichlet values on boundary points: nbor is MESH%NBOR
    (1-based), points with limdir == kdir take fbor.  sm and f (and the
    stored matrix) are modified in place; numpy arrays (host path) or torch
    CUDA tensors (device path)."""
    L = _native.lib()
    if _is_torch(sm):
        import torch
        dev = sm.device
        m = A.mesh
        nb = torch.as_tensor(np.ascontiguousarray(nbor, dtype=np.int32), device=dev)
        ld = torch.as_tensor(np.ascontiguousarray(limdir, dtype=np.int32), device=dev)
        fb = torch.as_tensor(fbor, dtype=torch.float64, device=dev).contiguous()
        nptfr = int(nb.numel())
        if ld.numel() != nptfr or fb.numel() != nptfr:
            raise ValueError("DIRI01: nbor, limdir and fbor must have NPTFR values each")
        st = L.bief_diri01_dev(m.handle, nptfr, _ptr(nb), _ptr(ld), int(kdir), _ptr(fb),
                               _dev(sm, m.npoin, m, "sm"), _dev(f, m.npoin, m, "f"),
                               None if maskpt is None else _dev(maskpt, m.npoin, m, "maskpt"),
                               _stream(sm))
    else:
        _host_vec(sm, A.mesh.npoin)
        _host_vec(f, A.mesh.npoin)
        nb = np.ascontiguousarray(nbor, dtype=np.int32)
        ld = np.ascontiguousarray(limdir, dtype=np.int32)
        fb = np.ascontiguousarray(fbor, dtype=np.float64)
        if ld.size != nb.size or fb.size != nb.size:
            raise ValueError("DIRI01: nbor, limdir and fbor must have NPTFR values each")
        mk = None if maskpt is None else _host_in(maskpt, A.mesh.npoin, "maskpt")
        st = L.bief_diri01(A.mesh.handle, int(nb.size), _ptr(nb), _ptr(ld), int(kdir), _ptr(fb),
                           _ptr(sm), _ptr(f), None if mk is None else _ptr(mk))
    _check(st, "DIRI01")
    return sm, f


def coef_grad(A, xc, yc, lam, x, grad):
    """grad[e] = -lam_e^T K_e x_e (device tensors)."""
    m = A.mesh
    _check(_native.lib().bief_wave_coef_grad_dev(
        m.handle, _dev(xc, m.npoin, m, "x coordinates"), _dev(yc, m.npoin, m, "y coordinates"),
        _dev(lam, m.npoin, m, "lam"), _dev(x, m.npoin, m, "x"), _dev(grad, m.nelem, m, "grad"),
        _stream(x)), "bief_wave_coef_grad_dev")
    return grad


def mass_diff_grad(A, xc, yc, u, v, lam, x, kind=12, xmul_dif=1.0):
    """(dL/du, dL/dv) for x = A(u, v)^-1 b assembled by
    Matrix.assemble_mass_diff (kind 11 or 12), given the adjoint lam
    (A^T lam = dL/dx); dL/dv is None for kind 11.  Device tensors."""
    import torch
    m = A.mesh
    if kind == 12 and v is None:
        raise ValueError("MATDIFUV needs v")
    gu = torch.empty_like(u)
    gv = torch.empty_like(u) if kind == 12 else None
    _check(_native.lib().bief_mass_diff_grad_dev(
        m.handle, _dev(xc, m.npoin, m, "x coordinates"), _dev(yc, m.npoin, m, "y coordinates"),
        float(xmul_dif), int(kind), _dev(u, m.npoin, m, "u"),
        None if v is None else _dev(v, m.npoin, m, "v"), _dev(lam, m.npoin, m, "lam"),
        _dev(x, m.npoin, m, "x"), _dev(gu, m.npoin, m, "gu"),
        None if gv is None else _dev(gv, m.npoin, m, "gv"), _stream(x)),
        "bief_mass_diff_grad_dev")
    return gu, gv


def _host_vec(a, n):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("host vectors must be contiguous float64 numpy arrays")
    if a.size != n:
        raise ValueError(f"vector of size {a.size}, expected NPOIN={n}")
