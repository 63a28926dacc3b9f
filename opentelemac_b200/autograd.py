"""Differentiable wave-equation solve for the TelApy-side Python layer.

    x = A(c)^-1 b,    A(c) = M + sum_e c_e K_e

with M the P1 mass matrix and K_e the unit-coefficient P1 stiffness matrix
of element e (the operator PROPAG assembles for the wave equation, with
c_e = dt*g*h_e).  `WaveSolve` is a torch.autograd.Function whose forward
assembles A(c) on the device (bief_assemble_wave_dev) and solves with the
library's GRACJG kernels; its backward solves the adjoint system
A^T lam = dL/dx with the same kernels (A is symmetric) and forms the
per-element gradient dL/dc_e = -lam_e^T K_e x_e in one element pass
(bief_wave_coef_grad_dev).  dL/db = lam.

`unrolled_loop` chains `nsteps` implicit steps x_{n+1} = A^-1 (M x_n) and
keeps only every `checkpoint_every`-th state: the steps in between are
recomputed during the backward pass (torch.utils.checkpoint), so memory is
O(nsteps / checkpoint_every) vectors instead of O(nsteps).

`MassDiffSolve` does the same for the operator in PROPAG's own form with
node coefficients (MATDIFUV with u = DM1 and v = HPROP, or MATDIF with u per
node; bief_assemble_mass_diff_dev) and returns dL/du and dL/dv per node
(bief_mass_diff_grad_dev): the gradient with respect to the depth field.

No reference counterpart (the reference's adjoint is a whole-model adjoint,
propag_adj.f:697, built on the same SOLVE).
"""
import torch
import torch.utils.checkpoint as tcp

from . import bief


class WaveProblem:
    """A mesh on the GPU with the two operators the loop needs: A(c)
    (re-assembled for each coefficient field) and the mass matrix M."""

    def __init__(self, x, y, ikle0, device="cuda", eps=1e-13, precon=2, nitmax=1000000):
        dev = torch.device(device)
        self.device = dev
        self.npoin = int(x.shape[0])
        self.nelem = int(ikle0.shape[0])
        self.xc = torch.as_tensor(x, dtype=torch.float64, device=dev).contiguous()
        self.yc = torch.as_tensor(y, dtype=torch.float64, device=dev).contiguous()
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        self.mesh_a = bief.Mesh(ikle0, self.npoin, device=idx)
        self.mesh_m = bief.Mesh(ikle0, self.npoin, device=idx)
        self.A = bief.Matrix(self.mesh_a)
        self.M = bief.Matrix(self.mesh_m)
        self.M.assemble_wave(self.xc, self.yc, torch.zeros(self.nelem, dtype=torch.float64,
                                                           device=dev))
        self.eps, self.precon, self.nitmax = eps, precon, nitmax
        self.solves = 0

    def cfg(self):
        return bief.SlvCfg(slv=1, nitmax=self.nitmax, precon=self.precon, krylov=0,
                           eps=self.eps, zero=0.0)

    def assemble(self, coef):
        """(Re-)assemble A(coef) on the device: one element pass, done before
        every solve so that the handle never holds a stale operator."""
        self.A.assemble_wave(self.xc, self.yc, coef.detach().contiguous())
        return self.A

    def solve(self, coef, b):
        A = self.assemble(coef)
        x = torch.zeros_like(b)
        st, nit, relres = bief.solve(x, A, b.detach().contiguous(), self.cfg())
        if st != 0:
            raise bief.BiefError(st, "wave solve did not converge")
        self.solves += 1
        return x

    def mass(self, v):
        out = torch.empty_like(v)
        bief.matvec("X=AY    ", out, self.M, v.detach().contiguous())
        return out

    def coef_grad(self, lam, x):
        g = torch.empty(self.nelem, dtype=torch.float64, device=self.device)
        bief.coef_grad(self.A, self.xc, self.yc, lam.contiguous(), x.contiguous(), g)
        return g

    def close(self):
        self.mesh_a.close()
        self.mesh_m.close()


class WaveSolve(torch.autograd.Function):
    """x = A(coef)^-1 b with gradients for coef and b."""

    @staticmethod
    def forward(ctx, coef, b, prob):
        x = prob.solve(coef, b)
        ctx.prob = prob
        ctx.save_for_backward(coef, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        coef, x = ctx.saved_tensors
        prob = ctx.prob
        lam = prob.solve(coef, gx)                 # adjoint: A^T = A
        gcoef = prob.coef_grad(lam, x) if ctx.needs_input_grad[0] else None
        gb = lam if ctx.needs_input_grad[1] else None
        return gcoef, gb, None


class MassMatvec(torch.autograd.Function):
    """v -> M v (M symmetric, so the backward is M g)."""

    @staticmethod
    def forward(ctx, v, prob):
        ctx.prob = prob
        return prob.mass(v)

    @staticmethod
    def backward(ctx, g):
        return ctx.prob.mass(g), None


def wave_solve(coef, b, prob):
    return WaveSolve.apply(coef, b, prob)


class MassDiffProblem:
    """The wave-equation operator in PROPAG's own form with node
    coefficients (propag.F:673-676,1407-1408):
        A(u, v) = MT01AA(xmul_mass) + MT02AA(xmul_dif; u, v)
    kind 12: MATDIFUV, u = DM1 and v = HPROP (the depth) per node, as
    PROPAG calls it with xmul_dif = -1; kind 11: MATDIF with u per node."""

    def __init__(self, x, y, ikle0, kind=12, xmul_mass=1.0, xmul_dif=-1.0, device="cuda",
                 eps=1e-13, precon=2, nitmax=1000000):
        if kind not in (11, 12):
            raise ValueError("kind 11 or 12")
        dev = torch.device(device)
        self.device = dev
        self.kind, self.xmul_mass, self.xmul_dif = kind, float(xmul_mass), float(xmul_dif)
        self.npoin = int(x.shape[0])
        self.xc = torch.as_tensor(x, dtype=torch.float64, device=dev).contiguous()
        self.yc = torch.as_tensor(y, dtype=torch.float64, device=dev).contiguous()
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        self.mesh = bief.Mesh(ikle0, self.npoin, device=idx)
        self.A = bief.Matrix(self.mesh)
        self.eps, self.precon, self.nitmax = eps, precon, nitmax
        self.solves = 0

    def assemble(self, u, v):
        self.A.assemble_mass_diff(self.xc, self.yc, u.detach().contiguous(),
                                  None if v is None else v.detach().contiguous(),
                                  kind=self.kind, xmul_mass=self.xmul_mass,
                                  xmul_dif=self.xmul_dif)
        return self.A

    def solve(self, u, v, b):
        A = self.assemble(u, v)
        x = torch.zeros_like(b)
        cfg = bief.SlvCfg(slv=1, nitmax=self.nitmax, precon=self.precon, krylov=0,
                          eps=self.eps, zero=0.0)
        st, nit, relres = bief.solve(x, A, b.detach().contiguous(), cfg)
        if st != 0:
            raise bief.BiefError(st, "wave solve did not converge")
        self.solves += 1
        return x

    def grad(self, u, v, lam, x):
        return bief.mass_diff_grad(self.A, self.xc, self.yc, u.detach().contiguous(),
                                   None if v is None else v.detach().contiguous(),
                                   lam.contiguous(), x.contiguous(), kind=self.kind,
                                   xmul_dif=self.xmul_dif)

    def close(self):
        self.mesh.close()


class MassDiffSolve(torch.autograd.Function):
    """x = A(u, v)^-1 b with gradients for the node coefficients u, v and
    for b: the adjoint solve A^T lam = dL/dx on the same kernels (A is
    symmetric), then dL/du, dL/dv summed per node over its elements."""

    @staticmethod
    def forward(ctx, u, v, b, prob):
        x = prob.solve(u, v, b)
        ctx.prob = prob
        ctx.has_v = v is not None
        ctx.save_for_backward(u, v if v is not None else u, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        u, v, x = ctx.saved_tensors
        v = v if ctx.has_v else None
        prob = ctx.prob
        lam = prob.solve(u, v, gx)
        gu = gv = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            gu, gv = prob.grad(u, v, lam, x)
        return (gu if ctx.needs_input_grad[0] else None,
                gv if ctx.needs_input_grad[1] else None,
                lam if ctx.needs_input_grad[2] else None, None)


def mass_diff_solve(u, v, b, prob):
    return MassDiffSolve.apply(u, v, b, prob)


def unrolled_loop(coef, x0, prob, nsteps=50, checkpoint_every=10):
    """x_{n+1} = A(coef)^-1 M x_n for n < nsteps; returns x_nsteps.  With
    checkpoint_every > 0 only every checkpoint_every-th state is kept for
    the backward pass and the others are recomputed."""
    def segment(x, c, k):
        for _ in range(k):
            x = WaveSolve.apply(c, MassMatvec.apply(x, prob), prob)
        return x

    x = x0
    n = 0
    while n < nsteps:
        k = min(checkpoint_every, nsteps - n) if checkpoint_every > 0 else nsteps - n
        if checkpoint_every > 0:
            x = tcp.checkpoint(segment, x, coef, k, use_reentrant=False)
        else:
            x = segment(x, coef, k)
        n += k
    return x
