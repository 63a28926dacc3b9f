"""Batched solve of many independent P1 meshes in one persistent launch.

The meshes become the diagonal blocks of one block-diagonal mesh (each
instance's nodes start on a multiple of 32); `bief_batch_solve_mixed_dev`
runs the mixed-precision algorithm on every instance at once with its own
scalars and convergence mask.  The work tile (1024 x nodes-per-thread nodes)
is chosen by a small autotuner that times a few inner iterations of each
candidate on the actual batch.
"""
import ctypes

import numpy as np

from . import _native, bief


class BatchSolver:
    def __init__(self, meshes, device=0):
        """meshes: list of (npoin, ikle0) with ikle0 (nelem, 3) 0-based."""
        import torch
        self.device = torch.device("cuda", device)
        self.ninst = len(meshes)
        if not 1 <= self.ninst <= 512:
            raise ValueError("1..512 instances")
        offs, n_list, e_off, ik_all = [], [], [], []
        off, eo = 0, 0
        for npoin, ik in meshes:
            offs.append(off)
            n_list.append(int(npoin))
            e_off.append(eo)
            ik_all.append(np.asarray(ik, dtype=np.int64) + off)
            eo += ik.shape[0]
            off += (int(npoin) + 31) // 32 * 32
        self.node_off = np.array(offs, dtype=np.int32)
        self.npoin = np.array(n_list, dtype=np.int32)
        self.elem_off = np.array(e_off + [eo], dtype=np.int64)
        self.total_nodes = off
        self.mesh = bief.Mesh(np.concatenate(ik_all).astype(np.int32), off, device=device)
        self.A = bief.Matrix(self.mesh)
        self.tuned_npt = None
        self.last = None

    # -- layout helpers
    def gather(self, vecs, fill=0.0):
        """Per-instance vectors -> one device vector over the whole mesh."""
        import torch
        out = torch.full((self.total_nodes,), fill, dtype=torch.float64, device=self.device)
        for k, v in enumerate(vecs):
            o, n = int(self.node_off[k]), int(self.npoin[k])
            out[o:o + n] = torch.as_tensor(v, dtype=torch.float64, device=self.device)
        return out

    def scatter(self, x):
        return [x[int(o):int(o) + int(n)] for o, n in zip(self.node_off, self.npoin)]

    def assemble_wave(self, xs, ys, coefs):
        """A_k = M_k + coef_e K_e for every instance (coordinates and per-
        element coefficients per instance)."""
        import torch
        xc, yc = self.gather(xs), self.gather(ys)
        coef = torch.cat([torch.as_tensor(c, dtype=torch.float64, device=self.device)
                          for c in coefs])
        self.A.assemble_wave(xc, yc, coef.contiguous())

    def set_segments(self, segs):
        """Segment storage (MATRIX STORAGE 3) for every instance: segs is one
        (g1, g2) pair of 0-based GLOSEG columns per instance, numbered as the
        instance's own mesh numbers them (meshgen.segments gives STOSEG's
        numbering).  The instances' segment lists are concatenated, so each
        node keeps its segments in its own instance's order; call
        to_segments() after assemble_wave() to convert the matrix."""
        if len(segs) != self.ninst:
            raise ValueError(f"{len(segs)} segment lists for {self.ninst} instances")
        g1 = np.concatenate([np.asarray(a, np.int64) + int(o) for (a, _), o in
                             zip(segs, self.node_off)])
        g2 = np.concatenate([np.asarray(b, np.int64) + int(o) for (_, b), o in
                             zip(segs, self.node_off)])
        self.mesh.set_segments(g1, g2)
        return self

    def to_segments(self):
        """ASSEX3 of the assembled EBE matrix into the instances' segments."""
        self.A.to_segments()
        return self

    # -- solve
    def solve_mixed(self, x, b, precon=2, inner_tol=1e-4, outer_tol=1e-8, max_outer=1000,
                    max_inner=1000000, nodes_per_thread=None, threads_per_block=None):
        """x (in/out), b: device vectors over the whole mesh.  Returns a dict
        of per-instance status, inner/outer counts, relres and kernel ms.
        Without nodes_per_thread the work tile and block shape come from
        the autotuner."""
        import torch
        if nodes_per_thread is None:
            nodes_per_thread, threads_per_block, _ = self.autotune(b, precon, inner_tol,
                                                                   outer_tol)
        if threads_per_block is None:
            threads_per_block = 1024
        ni = self.ninst
        st = np.zeros(ni, dtype=np.int32)
        outer = np.zeros(ni, dtype=np.int32)
        inner = np.zeros(ni, dtype=np.int32)
        relres = np.zeros(ni, dtype=np.float64)
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        s = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        rc = _native.lib().bief_batch_solve_mixed_dev(
            self.mesh.handle, ni, vp(self.node_off), vp(self.npoin),
            bief._dev(x, self.total_nodes, self.mesh, "x"),
            bief._dev(b, self.total_nodes, self.mesh, "b"), precon, inner_tol,
            outer_tol, max_outer, max_inner, nodes_per_thread, threads_per_block, vp(st),
            vp(outer), vp(inner), vp(relres), s)
        if rc < 0:
            raise bief.BiefError(rc, "batched solve")
        self.last = dict(status=st, outer=outer, inner=inner, relres=relres,
                         kernel_ms=self.mesh.last_timing()[0], nodes_per_thread=nodes_per_thread,
                         threads_per_block=threads_per_block)
        return self.last

    def autotune(self, b, precon=2, inner_tol=1e-4, outer_tol=1e-8, candidates=(1, 2, 4, 8),
                 block_shapes=(256, 512, 1024), residencies=(1, 2), probe_inner=30):
        """Pick (nodes per thread, threads per block, blocks per SM) by timing
        `probe_inner` inner iterations of every instance with each triple
        (kernel time per inner iteration of the longest-running instance).
        The triple is kept for later solves (the residency is set on the
        mesh); self.tune_table holds every candidate's time.  The batched
        dot order depends on none of the three but the nodes per thread and
        threads per block."""
        import torch
        if self.tuned_npt is not None:
            return self.tuned_npt
        best, best_t = None, None
        self.tune_table = {}
        for bps in residencies:
            self.mesh.set_blocks_per_sm(bps)
            for threads in block_shapes:
                for npt in candidates:
                    x = torch.zeros_like(b)
                    r = self.solve_mixed(x, b, precon, inner_tol, outer_tol, 1000, probe_inner,
                                         npt, threads)
                    per = r["kernel_ms"] / max(int(r["inner"].max()), 1)
                    self.tune_table[(npt, threads, bps)] = per
                    if best_t is None or per < best_t:
                        best, best_t = (npt, threads, bps), per
        self.mesh.set_blocks_per_sm(best[2])
        self.tuned_npt = best
        return best

    def close(self):
        self.mesh.close()
