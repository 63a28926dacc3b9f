// bief_kernels.cuh -- sm_100a kernels of the BIEF EBE P1 CG path.
//
//  k_matvec       MATVEC 'X=..AY' / 'X=..TAY' (matvec.f:316-380 ->
//                 mv0303.f:117-630 + assvec.f:88-93), node-centric gather
//                 straight from the EBE arrays.
//  k_precd1_*     PRECD1 change of variables (precd1.f:88-158, om1111.f:559-600).
//  k_build_rec    binary64 gather-ready records of the scaled operator.
//  k_build_seg32  binary32 edge-assembled copy of the scaled operator.
//  k_cg64         GRACJG (gracjg.F:169-420) as ONE persistent cooperative
//                 kernel: two grid reductions per iteration, fused vector
//                 updates, convergence tested on the device.
//  k_mixed        binary32 CG with binary64 reliable updates, one launch.
//  k_wave_*       on-device MT01AA + MT02AA + ASSVEC diagonal assembly.
//  k_coef_grad    per-element adjoint gradient -lambda_e^T K_e x_e.
#pragma once

#include "bief_device.cuh"

namespace bief {

// Shape of the persistent solver kernels: threads per block (one or more
// blocks per SM) and rows interleaved per thread in the gather phases.
// Every persistent kernel is also built for twice as many resident blocks
// per SM (MINB = 2 CG_MIN_BLOCKS: half the registers per thread, some of
// its state spilled to L1): twice the warps to hide memory latency when a
// solve streams its operator from HBM, at the price of the spills and of
// twice the blocks in every grid reduction.
#ifndef BIEF_CG_THREADS
#define BIEF_CG_THREADS 1024
#endif
#ifndef BIEF_ROW_ILP
#define BIEF_ROW_ILP 1
#endif
#ifndef BIEF_CG_MIN_BLOCKS
#define BIEF_CG_MIN_BLOCKS (1024 / BIEF_CG_THREADS)
#endif
constexpr int CG_THREADS = BIEF_CG_THREADS;
constexpr int CG_MIN_BLOCKS = BIEF_CG_MIN_BLOCKS;
constexpr int ROW_ILP = BIEF_ROW_ILP;

// ---------------------------------------------------------------------------
// MATVEC
// ---------------------------------------------------------------------------
enum : int { OP_AY = 0, OP_XPAY, OP_MAY, OP_XMAY, OP_XPCAY, OP_CAY };

template <int TD, bool SYM, bool TRANS>
__global__ void __launch_bounds__(256) k_matvec(int npoin, int nelem, const int *__restrict__ ptr,
                                                const int *__restrict__ ek, const int *__restrict__ ik,
                                                const double *__restrict__ xm,
                                                const double *__restrict__ da,
                                                const double *__restrict__ y, double *x, int opc,
                                                double c) {
  // OS combination of MESH%T into X (matvec.f:369-380, :329-340)
  auto store = [&](int i, double acc) {
    double r;
    switch (opc) {
      case OP_AY: r = acc; break;
      case OP_XPAY: r = add(x[i], acc); break;
      case OP_MAY: r = -acc; break;
      case OP_XMAY: r = sub(x[i], acc); break;
      case OP_XPCAY: r = add(x[i], mul(c, acc)); break;
      default: r = mul(c, acc); break;
    }
    x[i] = r;
  };
  auto vec = [&](int j) { return __ldg(y + j); };
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += stride)
    store(i, ebe_row<double, SYM, TRANS>(i, diag_term<TD>(__ldg(y + i), da, i), ptr, ek, ik, xm,
                                         nelem, vec));
}

// MATVEC from the gather records of the mesh (Mv16, built with the mesh):
// per entry, in the 32-node sliced layout, the element and local point and
// the element's two other vertices, so that the coefficient and the vertex
// loads of an entry depend on one coalesced index load only (ebe_row goes
// index -> IKLE -> vertex values) and IKLE is not read.  Three formats, the
// most compact the numbering allows:
//   MV_LOCAL  (IELEM - eb) << 2 | IDP-1 in 16 bits (eb: the slice's smallest
//             element) and the vertices as 16-bit offsets from the node: 6 B;
//   MV_BAND   IELEM << 2 | IDP-1 in 32 bits, 16-bit vertex offsets: 8 B;
//   MV_ANY    IELEM << 2 | IDP-1 and the two vertices, 32 bits each: 12 B
// (against 4 B of element index plus 8 B of IKLE read through it).  The
// index streams are loaded evict-first; the additions are ebe_row's, in its
// order, so the bits are the same.
enum : int { MV_NONE = 0, MV_LOCAL = 1, MV_BAND = 2, MV_ANY = 3 };

struct Mv16 {
  const unsigned char *deg;    // per node: gather entries
  const int *off;              // per slice: first record
  const int *eb;               // per slice: smallest element number (MV_LOCAL)
  const void *ek;              // per record: unsigned short (MV_LOCAL) or int
  const void *dv;              // per record: short2 offsets or int2 vertices (MV_ANY)
};

// Element, local point and the two other vertices of record r of node i.
template <int FMT>
__device__ __forceinline__ void mv_entry(const Mv16 &M, int i, int eb, int r, int &e, int &k,
                                         int &a, int &b) {
  int p;
  if constexpr (FMT == MV_LOCAL) {
    p = __ldcs(static_cast<const unsigned short *>(M.ek) + r);
    e = eb + (p >> 2);
  } else {
    p = __ldcs(static_cast<const int *>(M.ek) + r);
    e = p >> 2;
  }
  k = p & 3;
  if constexpr (FMT == MV_ANY) {
    const int2 v = __ldcs(static_cast<const int2 *>(M.dv) + r);
    a = v.x;
    b = v.y;
  } else {
    const short2 d = __ldcs(static_cast<const short2 *>(M.dv) + r);
    a = i + d.x;
    b = i + d.y;
  }
}

template <int NB, bool SYM, bool TRANS, int FMT, class V>
__device__ __forceinline__ void mv16_batch(double &acc, int i, int eb, int b0, int m,
                                           const Mv16 &M, const double *__restrict__ xm, int ne,
                                           V vec) {
  int e[NB], k[NB], va[NB], vb[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) mv_entry<FMT>(M, i, eb, b0 + 32 * (m + q), e[q], k[q], va[q], vb[q]);
  double xa[NB], xb[NB], ya[NB], yb[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int a = (k[q] == 2) ? 0 : k[q] + 1;  // (k+1) mod 3
    const int b = (k[q] == 0) ? 2 : k[q] - 1;  // (k+2) mod 3
    const int ca = TRANS ? xm_col<SYM>(a, k[q]) : xm_col<SYM>(k[q], a);
    const int cb = TRANS ? xm_col<SYM>(b, k[q]) : xm_col<SYM>(k[q], b);
    xa[q] = __ldg(xm + (size_t)ca * ne + e[q]);
    xb[q] = __ldg(xm + (size_t)cb * ne + e[q]);
    ya[q] = vec(va[q]);
    yb[q] = vec(vb[q]);
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) acc = add(acc, add(mul(xa[q], ya[q]), mul(xb[q], yb[q])));
}

// Gather entries per batch of k_matvec16 (all index loads of a batch, then
// all coefficient and vertex loads, then the additions in order).
#ifndef BIEF_MV16_BATCH
#define BIEF_MV16_BATCH 4
#endif
constexpr int MV16_B = BIEF_MV16_BATCH;
// Threads per block of k_matvec16 (one node each): 128 measured 84.0 µs
// against 85.5-86.0 with 256 at 4.0M nodes, equal at 1.0M.
#ifndef BIEF_MV16_THREADS
#define BIEF_MV16_THREADS 128
#endif
constexpr int MV16_T = BIEF_MV16_THREADS;

template <int TD, bool SYM, bool TRANS, int FMT>
__global__ void __launch_bounds__(MV16_T) k_matvec16(int npoin, int nelem, Mv16 M,
                                                  const double *__restrict__ xm,
                                                  const double *__restrict__ da,
                                                  const double *__restrict__ y, double *x, int opc,
                                                  double c) {
  auto vec = [&](int j) { return __ldg(y + j); };
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += stride) {
    const int deg = __ldcs(M.deg + i);
    const int b0 = __ldg(M.off + (i >> 5)) + (i & 31);
    const int eb = FMT == MV_LOCAL ? __ldg(M.eb + (i >> 5)) : 0;
    double acc = TD == DIA_Q ? mul(__ldg(y + i), __ldcs(da + i)) : diag_term<TD>(__ldg(y + i), da, i);
    int m = 0;
    for (; m + MV16_B <= deg; m += MV16_B)
      mv16_batch<MV16_B, SYM, TRANS, FMT>(acc, i, eb, b0, m, M, xm, nelem, vec);
    if constexpr (MV16_B / 2 > 1) {
      if (m + MV16_B / 2 <= deg) {
        mv16_batch<MV16_B / 2, SYM, TRANS, FMT>(acc, i, eb, b0, m, M, xm, nelem, vec);
        m += MV16_B / 2;
      }
    }
    for (; m < deg; ++m) mv16_batch<1, SYM, TRANS, FMT>(acc, i, eb, b0, m, M, xm, nelem, vec);
    double r;  // OS combination of MESH%T into X (matvec.f:369-380, :329-340)
    switch (opc) {
      case OP_AY: r = acc; break;
      case OP_XPAY: r = add(x[i], acc); break;
      case OP_MAY: r = -acc; break;
      case OP_XMAY: r = sub(x[i], acc); break;
      case OP_XPCAY: r = add(x[i], mul(c, acc)); break;
      default: r = mul(c, acc); break;
    }
    x[i] = r;
  }
}

// MATVEC 'X=AY' in binary32 (no reference counterpart) on the binary32
// edge-assembled copy of the operator, the product of the binary32 inner CG:
// X_i = s_i Y_i + sum_j c_ij (Y_j - Y_i), with s_i the row sum and c_ij the
// assembled off-diagonal coefficients, slots in sliced order (C16: their
// neighbours as 16-bit offsets).
template <bool C16>
__global__ void __launch_bounds__(256) k_matvec32(int npoin, Sell S, const float *__restrict__ y,
                                                  float *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    float a0, a1;
    seg_row2<C16>(i, i, false, __ldg(y + i), 0.0f, a0, a1, S,
                  [&](int k) { return __ldg(y + k); });
    x[i] = a0;
  }
}

// ---------------------------------------------------------------------------
// Segment storage (STO=3).  Per node, one slot per incident segment in
// ascending segment order (sliced layout: slot m of node i at
// off[i/32] + 32m + i%32): sx = ISEG<<1 | side (side 0: node is GLOSEG1,
// side 1: GLOSEG2), col = the other end.  XA is XA(NSEG) ('S') or
// XA(NSEG,2) ('Q', second column from NSEG on).
// ---------------------------------------------------------------------------

// MVSEG (mvseg.f:110-720): X takes the diagonal term through OV
// (ov.f:177-324: 'X=YZ', 'X=CYZ' = (C*Y)*Z, 'X=X+YZ', ...), then for each
// incident segment in ascending order X = X +/- [C*]XA*Y(other), the
// additions the reference's segment loop makes into this node, in its order.
template <int TD, bool SYM, bool TRANS>
__global__ void __launch_bounds__(256) k_mvseg(int npoin, int nseg, bool ext,
                                               const int *__restrict__ meta,
                                               const int *__restrict__ off,
                                               const int *__restrict__ sx,
                                               const int *__restrict__ col,
                                               const double *__restrict__ xa,
                                               const double *__restrict__ da,
                                               const double *__restrict__ y, double *x, int opc,
                                               double c) {
  const bool neg = (opc == OP_MAY || opc == OP_XMAY);
  const bool cm = (opc == OP_CAY || opc == OP_XPCAY);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const double yi = __ldg(y + i);
    double r;
    if (TD == DIA_0) {
      // 'X=C' with 0 for X=AY, X=CAY, X=-AY; nothing for the X=X+.. forms
      r = (opc == OP_AY || opc == OP_CAY || opc == OP_MAY) ? 0.0 : x[i];
    } else {
      const double d = TD == DIA_Q ? mul(yi, __ldg(da + i)) : yi;
      const double cd = TD == DIA_Q ? mul(mul(c, yi), __ldg(da + i)) : mul(c, yi);
      switch (opc) {
        case OP_AY: r = d; break;
        case OP_CAY: r = cd; break;
        case OP_MAY: r = -d; break;
        case OP_XPAY: r = add(x[i], d); break;
        case OP_XMAY: r = sub(x[i], d); break;
        default: r = add(x[i], cd); break;
      }
    }
    if (ext) {
      const int deg = __ldg(meta + i) & 0xffff;
      const int base = __ldg(off + (i >> 5)) + (i & 31);
      for (int m = 0; m < deg; ++m) {
        const int p = __ldg(sx + base + 32 * m);
        const int j = __ldg(col + base + 32 * m);
        const int q = SYM ? 0 : ((p & 1) ^ (TRANS ? 1 : 0));
        double a = __ldg(xa + (size_t)q * nseg + (p >> 1));
        if (cm) a = mul(c, a);
        const double t = mul(a, __ldg(y + j));
        r = neg ? sub(r, t) : add(r, t);
      }
    }
    x[i] = r;
  }
}

// OMSEG 'M=DMD' off-diagonal part (omseg.f:530-541):
// XA(ISEG) * D(GLOSEG1) * D(GLOSEG2), for each stored column.
__global__ void k_precd1_segs(int nseg, int ncol, const int *__restrict__ g1,
                              const int *__restrict__ g2, const double *__restrict__ dsc,
                              const double *__restrict__ xa, double *xas) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
    const double d1 = dsc[g1[s]], d2 = dsc[g2[s]];
    for (int q = 0; q < ncol; ++q)
      xas[(size_t)q * nseg + s] = mul(mul(xa[(size_t)q * nseg + s], d1), d2);
  }
}

// Per slot, the binary64 coefficient of the working operator's 'X=AY' row:
// XA1 for side 0, XA2 for side 1.
template <bool SYM, bool TRANS = false>
__global__ void k_build_sgc(int npoin, int nseg, const int *__restrict__ meta,
                            const int *__restrict__ off, const int *__restrict__ sx,
                            const double *__restrict__ xa, double *sg_c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const int deg = meta[i] & 0xffff;
    const int base = off[i >> 5] + (i & 31);
    for (int m = 0; m < deg; ++m) {
      const int p = sx[base + 32 * m];
      sg_c[base + 32 * m] = xa[(size_t)(SYM ? 0 : ((p & 1) ^ (TRANS ? 1 : 0))) * nseg + (p >> 1)];
    }
  }
}

// Binary32 operator of a symmetric segment matrix for the mixed solver: the
// slot coefficients rounded, and the row sum diag + XA of each slot added
// in slot order in binary64, rounded once.
template <int TD>
__global__ void k_build_sg32(int npoin, const int *__restrict__ meta, const int *__restrict__ off,
                             const double *__restrict__ sg_c, const double *__restrict__ da,
                             float *seg_c, float *s32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const int deg = meta[i] & 0xffff;
    const int base = off[i >> 5] + (i & 31);
    double srow = TD == DIA_Q ? da[i] : (TD == DIA_I ? 1.0 : 0.0);
    for (int m = 0; m < deg; ++m) {
      const double cv = sg_c[base + 32 * m];
      seg_c[base + 32 * m] = (float)cv;
      srow = add(srow, cv);
    }
    s32[i] = (float)srow;
  }
}

// ASSEX3 for P1 (assex3.f:150-160 -> as3_1111_s.f:71-79, as3_1111_q.f:85-98,
// STOXMT=1): each segment sums, from zero and in element order, the EBE
// terms of the (at most two) element faces that it is: face 1 (points 1-2)
// XMT(,1) [Q: and XMT(,4)], face 2 (2-3) XMT(,3) [XMT(,6)], face 3 (3-1)
// XMT(,2) [XMT(,5)].  For 'Q' the term of row IKLE(f) goes to column
// ORISEG (1 when GLOSEG1 = IKLE(f)) and the other to column 3-ORISEG.
// segel: per segment, its faces (e<<2 | f) in element order, -1 if none.
template <bool SYM>
__global__ void k_assex3(int nseg, int nelem, int ld, const int2 *__restrict__ segel,
                         const int *__restrict__ g1, const int *__restrict__ ik,
                         const double *__restrict__ xmt, double *xa) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
    const int2 fe = segel[s];
    double a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int p = q == 0 ? fe.x : fe.y;
      if (p < 0) continue;
      const int e = p >> 2, f = p & 3;
      if (SYM) {
        const int cs = f == 0 ? 0 : (f == 1 ? 2 : 1);
        a1 = add(a1, xmt[(size_t)cs * ld + e]);
      } else {
        const int ca = f == 0 ? 0 : (f == 1 ? 2 : 4);   // row IKLE(f)
        const int cb = f == 0 ? 3 : (f == 1 ? 5 : 1);   // row IKLE(f+1)
        const double va = xmt[(size_t)ca * ld + e], vb = xmt[(size_t)cb * ld + e];
        if (ik[(size_t)f * nelem + e] == g1[s]) {
          a1 = add(a1, va);
          a2 = add(a2, vb);
        } else {
          a2 = add(a2, va);
          a1 = add(a1, vb);
        }
      }
    }
    xa[s] = a1;
    if (!SYM) xa[(size_t)nseg + s] = a2;
  }
}

// DIRI01 (diri01.f:90-130, DIRAUX diraux.f:70-85) on boundary numbering:
// the Dirichlet values scattered to their nodes, SM corrected, the rows and
// columns of the Dirichlet nodes masked.  nbor is 1-based (MESH%NBOR).
// NBOR entries outside 1..NPOIN are skipped and flagged in *err.
__global__ void k_diri_scatter(int nptfr, int npoin, const int *__restrict__ nbor,
                               const int *__restrict__ limdir, int kdir,
                               const double *__restrict__ fbor, double *w1, int *err) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nptfr; k += gridDim.x * blockDim.x)
    if (limdir[k] == kdir) {
      const int n = nbor[k];
      if (n < 1 || n > npoin) {
        atomicExch(err, 1);
        continue;
      }
      w1[n - 1] = fbor[k];
    }
}

// SM = SM - W2 ('X=X-Y'), then W2 = 1 ('X=C')
__global__ void k_diri_nodes(int npoin, double *sm, double *w2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    sm[i] = sub(sm[i], w2[i]);
    w2[i] = 1.0;
  }
}

__global__ void k_diri_aux(int nptfr, int npoin, const int *__restrict__ nbor,
                           const int *__restrict__ limdir, int kdir,
                           const double *__restrict__ fbor, const double *__restrict__ dm,
                           double *sm, double *w2, double *f) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nptfr; k += gridDim.x * blockDim.x)
    if (limdir[k] == kdir) {
      const int n = nbor[k] - 1;
      if (n < 0 || n >= npoin) continue;   // flagged by k_diri_scatter
      sm[n] = mul(dm[n], fbor[k]);
      w2[n] = 0.0;
      f[n] = fbor[k];
    }
}

__global__ void k_diri_mask(int npoin, const double *__restrict__ mask, double *sm, double *f,
                            double *w2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    sm[i] = mul(sm[i], mask[i]);
    f[i] = mul(f[i], mask[i]);
    w2[i] = mul(w2[i], mask[i]);
  }
}

// Self-test of the bounded waits: one block enters a grid barrier one
// arrival short (as if another block never came), so its wait must give up
// after timeout_ns and record ST_TIMEOUT instead of hanging.
__global__ void k_selftest_wait(Ctl *ctl, long long timeout_ns) {
  int nbar = 1;
  grid_barrier(ctl, timeout_ns, nbar);
}

// ---------------------------------------------------------------------------
// PRECD1 change of variables, DIADON=.FALSE., PREXSM=.TRUE.
// Node part: D = A%D; [|D|]; D = SQRT(D); X = X*D; D = 1/D guarded
// (ovd.f:92-102: |D| > 1e-10 ? 1/D : 1.0); diagonal of D.A.D
// (om1111.f:561-570: 'Q' -> DM*D*D, 'I' -> D*D); B = B*D.
// ---------------------------------------------------------------------------
__global__ void k_precd1_nodes(int npoin, int precon, int td_in, const double *__restrict__ dm,
                               double *x, const double *b_in, double *b_out, double *dsc,
                               double *dms) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    double d = dm[i];
    if (precon == 5) d = fabs(d);
    d = __dsqrt_rn(d);
    x[i] = mul(x[i], d);
    d = (fabs(d) > 1.0e-10) ? __ddiv_rn(1.0, d) : 1.0;
    dsc[i] = d;
    if (td_in == DIA_Q) {
      dms[i] = mul(mul(dm[i], d), d);
    } else if (td_in == DIA_I) {
      dms[i] = mul(d, d);
    } else {
      dms[i] = dm[i];
    }
    b_out[i] = mul(b_in[i], d);
  }
}

// Off-diagonal part of OM1111 'M=DMD' (om1111.f:589-600):
// XM(e,1)*D(i2)*D(i1), XM(e,2)*D(i3)*D(i1), XM(e,3)*D(i3)*D(i2) (and the
// same for columns 4..6 of 'Q' storage).
__global__ void k_precd1_elems(int nelem, int ndiag, const int *__restrict__ ik,
                               const double *__restrict__ dsc, const double *__restrict__ xm,
                               double *xms) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    const double d1 = dsc[ik[e]], d2 = dsc[ik[(size_t)nelem + e]],
                 d3 = dsc[ik[2 * (size_t)nelem + e]];
    for (int c = 0; c < ndiag; ++c) {
      const int cc = c % 3;
      const double da = cc == 0 ? d2 : d3;
      const double db = cc == 2 ? d2 : d1;
      xms[(size_t)c * nelem + e] = mul(mul(xm[(size_t)c * nelem + e], da), db);
    }
  }
}

// ---------------------------------------------------------------------------
// Gather-ready layouts of the working operator (see Sell in bief_device.cuh)
// ---------------------------------------------------------------------------
// TRANS: the coefficients of the transposed operator, XA(a,k) and XA(b,k)
// (mv0303.f 'X=TAY'), for the same two neighbours.
template <bool SYM, bool TRANS = false>
__global__ void k_build_rec(int npoin, int nelem, const int *__restrict__ ptr,
                            const int *__restrict__ ek, const double *__restrict__ xm,
                            const int *__restrict__ rec_off, double2 *rec_c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const int j0 = ptr[i], deg = ptr[i + 1] - j0;
    const int base = rec_off[i >> 5] + (i & 31);
    for (int m = 0; m < deg; ++m) {
      const int p = ek[j0 + m], e = p >> 2, k = p & 3;
      const int a = (k == 2) ? 0 : k + 1, b = (k == 0) ? 2 : k - 1;
      const int ca = TRANS ? xm_col<SYM>(a, k) : xm_col<SYM>(k, a);
      const int cb = TRANS ? xm_col<SYM>(b, k) : xm_col<SYM>(k, b);
      rec_c[base + 32 * m] = make_double2(xm[(size_t)ca * nelem + e], xm[(size_t)cb * nelem + e]);
    }
  }
}

// Binary32 edge-assembled operator: per node, slot coefficients and the row
// sum accumulated in binary64 in gather order, rounded once (symmetric
// storage).  rec_slot holds, per record, the slots of its two neighbours.
constexpr int MAX_NEIGHBOURS = 64;

template <int TD>
__global__ void k_build_seg32(int npoin, int nelem, const int *__restrict__ ptr,
                              const int *__restrict__ ek, const double *__restrict__ xm,
                              const double *__restrict__ da, const int *__restrict__ meta,
                              const int *__restrict__ rec_off,
                              const uchar2 *__restrict__ rec_slot,
                              const int *__restrict__ seg_off, float *seg_c, float *s32) {
  double c64[MAX_NEIGHBOURS];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const int j0 = ptr[i], deg = ptr[i + 1] - j0, nnb = meta[i] >> 16;
    const int rb = rec_off[i >> 5] + (i & 31), sb = seg_off[i >> 5] + (i & 31);
    for (int q = 0; q < nnb; ++q) c64[q] = 0.0;
    double s = TD == DIA_Q ? da[i] : (TD == DIA_I ? 1.0 : 0.0);
    for (int m = 0; m < deg; ++m) {
      const int p = ek[j0 + m], e = p >> 2, k = p & 3;
      const int a = (k == 2) ? 0 : k + 1, b = (k == 0) ? 2 : k - 1;
      const double xa = xm[(size_t)(k + a - 1) * nelem + e];
      const double xb = xm[(size_t)(k + b - 1) * nelem + e];
      const uchar2 sl = rec_slot[rb + 32 * m];
      c64[sl.x] = add(c64[sl.x], xa);
      c64[sl.y] = add(c64[sl.y], xb);
      s = add(s, add(xa, xb));
    }
    for (int q = 0; q < nnb; ++q) seg_c[sb + 32 * q] = (float)c64[q];
    s32[i] = (float)s;
  }
}

// ---------------------------------------------------------------------------
// GRACJG as a persistent kernel.
// ---------------------------------------------------------------------------
struct CgP {
  int npoin, nitmax;
  double eps;
  Sell S;                 // records of the working (scaled) operator
  const double *da;       // working diagonal
  const double *dsc;      // change of variables to undo (nullptr: none)
  double *x;
  const double *b;
  double *r, *d0, *d1, *ad;
  double *part;
  Ctl *ctl;
  long long timeout_ns;
};

// COMP: MODASS = 3, every P_DOTS a compensated dot (Dot2, dot_comp.f) in
// the device order (grid_reduce_comp); the vector operations are unchanged
// (their compensated forms in the reference only fill error vectors that
// GRACJG does not read).
template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_cg64(CgP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *r = P.r, *ad = P.ad;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  double s, red;
  CPair cs{0.0, 0.0};
  int nbar = 0;
  auto dot0 = [&]() {
    s = 0.0;
    cs = CPair{0.0, 0.0};
  };
  auto dacc = [&](double u, double v) {
    if constexpr (COMP)
      cdot_add(cs, u, v);
    else
      s = add(s, mul(u, v));
  };
  auto dred = [&](double &out) -> bool {
    if constexpr (COMP)
      return grid_reduce_comp(P.ctl, P.part, P.timeout_ns, nbar, cs, &out);
    else
      return grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &out, nullptr);
  };

  auto finish = [&](int status, int m, double rmrm, double xl, int relat) {
    if (P.dsc)  // solve.f:637-641: X = X*D
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = m;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rmrm, xl));
      P.ctl->relat = relat;
    }
  };

  // XL = P_DOTS(B,B) (gracjg.F:189)
  dot0();
  for (int i = lo + t; i < hi; i += T) dacc(b[i], b[i]);
  if (!dred(red)) return;
  double xl = red;
  if (__dsqrt_rn(xl) < 1.0e-15) {  // gracjg.F:194-202: X = 0
    for (int i = lo + t; i < hi; i += T) x[i] = 0.0;
    finish(ST_OK, 0, 0.0, 1.0, 0);
    return;
  }
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }  // gracjg.F:204-209
  const double tol = mul(xl, mul(P.eps, P.eps));

  // R = A X - B (gracjg.F:213-216)
  dot0();
  for (int i = lo + t; i < hi; i += ROW_ILP * T) {
    const int i1 = i + T;
    const bool h1 = ROW_ILP == 2 && i1 < hi;
    double a0 = diag_term<TD>(x[i], da, i), a1 = h1 ? diag_term<TD>(x[i1], da, i1) : 0.0;
    op_row2<STO>(i, i1, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double r0 = sub(a0, b[i]);
    r[i] = r0;
    dacc(r0, r0);
    if (h1) {
      const double r1 = sub(a1, b[i1]);
      r[i1] = r1;
      dacc(r1, r1);
    }
  }
  if (!dred(red)) return;
  double rmrm = red, rmgm = rmrm;
  if (isnan(rmrm)) { finish(ST_NAN, 0, rmrm, xl, relat); return; }
  if (rmrm < mul(mul(P.eps, P.eps), xl)) { finish(ST_OK, 0, rmrm, xl, relat); return; }

  // D = G (= R), AD = A D, DAD, RO (gracjg.F:248-261)
  double *cur = P.d0, *nxt = P.d1;
  dot0();
  for (int i = lo + t; i < hi; i += ROW_ILP * T) {
    const int i1 = i + T;
    const bool h1 = ROW_ILP == 2 && i1 < hi;
    const double d0 = r[i], d1 = h1 ? r[i1] : 0.0;
    cur[i] = d0;
    if (h1) cur[i1] = d1;
    double a0 = diag_term<TD>(d0, da, i), a1 = h1 ? diag_term<TD>(d1, da, i1) : 0.0;
    op_row2<STO>(i, i1, h1, a0, a1, P.S, [&](int j) { return r[j]; });
    ad[i] = a0;
    dacc(d0, a0);
    if (h1) {
      ad[i1] = a1;
      dacc(d1, a1);
    }
  }
  if (!dred(red)) return;
  double dad = red;
  if (!(dad > 0.0)) { finish(isnan(dad) ? ST_NAN : ST_BREAKDOWN, 0, rmrm, xl, relat); return; }
  double ro = __ddiv_rn(rmgm, dad);

  for (int m = 1;; ++m) {
    // X = X - RO*D (gracjg.F:268 / :387) fused with R = R - RO*AD (:290)
    // and RMRM = P_DOTS(R,R) (:295)
    const double nro = -ro;
    dot0();
    for (int i = lo + t; i < hi; i += T) {
      x[i] = add(x[i], mul(nro, cur[i]));
      const double ri = add(r[i], mul(nro, ad[i]));
      r[i] = ri;
      dacc(ri, ri);
    }
    if (!dred(red)) return;
    const double rm1gm1 = rmgm;
    rmrm = red;
    rmgm = rmrm;
    if (isnan(rmrm)) { finish(ST_NAN, m, rmrm, xl, relat); return; }
    if (rmrm <= tol) { finish(ST_OK, m, rmrm, xl, relat); return; }  // :303
    const double beta = __ddiv_rn(rmgm, rm1gm1);                       // :357

    // D = R + BETA*D (:361) computed where it is needed, AD = A D (:376),
    // DAD = P_DOTS(D,AD) (:382).  Every thread that needs D at node j
    // recomputes R(j)+BETA*D(j) from the previous direction, which gives
    // the same bits as the owner's value; the owner also stores it.
    dot0();
    for (int i = lo + t; i < hi; i += ROW_ILP * T) {
      const int i1 = i + T;
      const bool h1 = ROW_ILP == 2 && i1 < hi;
      const double d0 = add(r[i], mul(beta, cur[i]));
      const double d1 = h1 ? add(r[i1], mul(beta, cur[i1])) : 0.0;
      nxt[i] = d0;
      if (h1) nxt[i1] = d1;
      double a0 = diag_term<TD>(d0, da, i), a1 = h1 ? diag_term<TD>(d1, da, i1) : 0.0;
      op_row2<STO>(i, i1, h1, a0, a1, P.S, [&](int j) { return add(r[j], mul(beta, cur[j])); });
      ad[i] = a0;
      dacc(d0, a0);
      if (h1) {
        ad[i1] = a1;
        dacc(d1, a1);
      }
    }
    if (!dred(red)) return;
    dad = red;
    if (!(dad > 0.0)) { finish(isnan(dad) ? ST_NAN : ST_BREAKDOWN, m, rmrm, xl, relat); return; }
    ro = __ddiv_rn(rmgm, dad);  // :383 (RMDM = RMGM)
    double *tmp = cur; cur = nxt; nxt = tmp;

    if (m >= P.nitmax) {  // :406 -- last X update, then stop unconverged
      const double nr = -ro;
      for (int i = lo + t; i < hi; i += T) x[i] = add(x[i], mul(nr, cur[i]));
      finish(m, m, rmrm, xl, relat);
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// EQUNOR (equnor.f:106-311): CG on the normal equations A^T A x = A^T b,
// without preconditioning matrices (G aliases R), as ONE persistent kernel
// with three grid reductions per iteration.  P.S describes the working
// operator A, P.St its transpose (same neighbours, transposed
// coefficients); P.t holds A^T R.  As in k_cg64 the new direction
// D = BETA*D + A^T R is recomputed wherever it is needed, with the owner's
// bits.
// ---------------------------------------------------------------------------
struct EqP {
  int npoin, nitmax;
  double eps;
  Sell S, St;
  const double *da, *dsc;
  double *x;
  const double *b;
  double *r, *d0, *d1, *ad, *t;
  double *part;
  Ctl *ctl;
  long long timeout_ns;
};

template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_equnor(EqP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *r = P.r, *ad = P.ad, *atr = P.t;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  DotAcc<COMP, 1> s;
  double red;
  int nbar = 0;
  const bool h1 = false;

  auto finish = [&](int status, int m, double rmrm, double xl, int relat) {
    if (P.dsc)  // solve.f:637-641: X = X*D
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = m;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rmrm, xl));
      P.ctl->relat = relat;
    }
  };
  double a1 = 0.0;

  // XL = P_DOTS(B,B), absolute mode below 1 (equnor.f:108-114)
  s.zero();
  for (int i = lo + t; i < hi; i += T) s.acc(0, b[i], b[i]);
  if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
  double xl = red;
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }
  const double tol = mul(xl, mul(P.eps, P.eps));

  // R = A X - B, RMRM (:118-123)
  s.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(x[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double r0 = sub(a0, b[i]);
    r[i] = r0;
    s.acc(0, r0, r0);
  }
  if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
  double rmrm = red;
  if (isnan(rmrm)) { finish(ST_NAN, 0, rmrm, xl, relat); return; }
  if (rmrm < mul(mul(P.eps, P.eps), xl)) { finish(ST_OK, 0, rmrm, xl, relat); return; }  // :127

  // D = A^T R, TGMTGM (:160-163)
  double *cur = P.d0, *nxt = P.d1;
  s.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(r[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.St, [&](int j) { return r[j]; });
    cur[i] = a0;
    s.acc(0, a0, a0);
  }
  if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
  double tg = red;
  // AD = A D, ADAD, RO (:169-189)
  s.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(cur[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return cur[j]; });
    ad[i] = a0;
    s.acc(0, a0, a0);
  }
  if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
  double adad = red;
  if (!(adad > 0.0)) { finish(isnan(adad) ? ST_NAN : ST_BREAKDOWN, 0, rmrm, xl, relat); return; }
  double ro = __ddiv_rn(tg, adad);

  for (int m = 1;; ++m) {
    // X = X - RO D (:195 / :278), R = R - RO AD (:207), RMRM (:211)
    const double nro = -ro;
    s.zero();
    for (int i = lo + t; i < hi; i += T) {
      x[i] = add(x[i], mul(nro, cur[i]));
      const double ri = add(r[i], mul(nro, ad[i]));
      r[i] = ri;
      s.acc(0, ri, ri);
    }
    if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
    rmrm = red;
    if (isnan(rmrm)) { finish(ST_NAN, m, rmrm, xl, relat); return; }
    if (rmrm <= tol) { finish(ST_OK, m, rmrm, xl, relat); return; }  // :215

    // A^T R (:240), TGMTGM (:244)
    s.zero();
    for (int i = lo + t; i < hi; i += T) {
      double a0 = diag_term<TD>(r[i], da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.St, [&](int j) { return r[j]; });
      atr[i] = a0;
      s.acc(0, a0, a0);
    }
    if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
    const double tg1 = tg;
    tg = red;
    const double beta = __ddiv_rn(tg, tg1);  // :245

    // D = BETA D + A^T R (:247-250) where needed, AD = A D (:256), ADAD (:272)
    s.zero();
    for (int i = lo + t; i < hi; i += T) {
      const double di = add(mul(beta, cur[i]), atr[i]);
      nxt[i] = di;
      double a0 = diag_term<TD>(di, da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return add(mul(beta, cur[j]), atr[j]); });
      ad[i] = a0;
      s.acc(0, a0, a0);
    }
    if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
    adad = red;
    if (!(adad > 0.0)) { finish(isnan(adad) ? ST_NAN : ST_BREAKDOWN, m, rmrm, xl, relat); return; }
    ro = __ddiv_rn(tg, adad);  // :274
    double *tmp = cur; cur = nxt; nxt = tmp;

    if (m >= P.nitmax) {  // :280 -- last X update, then stop unconverged
      const double nr = -ro;
      for (int i = lo + t; i < hi; i += T) x[i] = add(x[i], mul(nr, cur[i]));
      finish(m, m, rmrm, xl, relat);
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// RESCJG (rescjg.f:134-315, conjugate residual) and ERRMIN (errmin.f:116-259,
// minimum error) without preconditioning matrices (G aliases R), each as ONE
// persistent kernel.  Same parameter block; ERRMIN also uses St (the
// transposed operator) and t (A^T R); the new ERRMIN direction is recomputed
// at every node that reads it (d0/d1 double-buffered).
// ---------------------------------------------------------------------------
struct Kry2P {
  int npoin, nitmax;
  double eps;
  Sell S, St;
  const double *da, *dsc;
  double *x;
  const double *b;
  double *r, *d0, *d1, *ad, *ag;
  double *part;
  Ctl *ctl;
  long long timeout_ns;
};

template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_rescjg(Kry2P P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *r = P.r, *d = P.d0, *ad = P.ad, *ag = P.ag;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  DotAcc<COMP, 2> sd;
  double rd[2];
  int nbar = 0;
  const bool h1 = false;
  double a1 = 0.0;
  auto finish = [&](int status, int m, double rmrm, double xl, int relat) {
    if (P.dsc)
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = m;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rmrm, xl));
      P.ctl->relat = relat;
    }
  };
  sd.zero();
  for (int i = lo + t; i < hi; i += T) sd.acc(0, b[i], b[i]);
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double xl = rd[0];
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }
  const double tol = mul(xl, mul(P.eps, P.eps));
  // R = A X - B, RMRM (:144-149)
  sd.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(x[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double ri = sub(a0, b[i]);
    r[i] = ri;
    sd.acc(0, ri, ri);
  }
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double rmrm = rd[0];
  if (isnan(rmrm)) { finish(ST_NAN, 0, rmrm, xl, relat); return; }
  if (rmrm < mul(mul(P.eps, P.eps), xl)) { finish(ST_OK, 0, rmrm, xl, relat); return; }
  // D = R, AD = A D, D.AD and AD.AD (:178-217)
  sd.zero();
  for (int i = lo + t; i < hi; i += T) {
    const double di = r[i];
    double a0 = diag_term<TD>(di, da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return r[j]; });
    d[i] = di;
    ad[i] = a0;
    sd.acc(0, di, a0);
    sd.acc(1, a0, a0);
  }
  if (!dred<COMP, 2>(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double adad = rd[1];
  double ro = __ddiv_rn(rd[0], adad);
  for (int m = 1;; ++m) {
    // X = X - RO D (:223 / :313), R = R - RO AD (:235), RMRM (:239)
    const double nro = -ro;
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      x[i] = add(x[i], mul(nro, d[i]));
      const double ri = add(r[i], mul(nro, ad[i]));
      r[i] = ri;
      sd.acc(0, ri, ri);
    }
    if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    rmrm = rd[0];
    if (isnan(rmrm)) { finish(ST_NAN, m, rmrm, xl, relat); return; }
    if (rmrm <= tol) { finish(ST_OK, m, rmrm, xl, relat); return; }  // :243
    // AG = A R (:258), AG.AD (:267)
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      double a0 = diag_term<TD>(r[i], da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return r[j]; });
      ag[i] = a0;
      sd.acc(0, a0, ad[i]);
    }
    if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    const double beta = __ddiv_rn(-rd[0], adad);  // :269
    // D = BETA D + R, AD = BETA AD + AG (:271-279), R.AD, AD.AD (:303-307)
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      d[i] = add(mul(beta, d[i]), r[i]);
      const double adi = add(mul(beta, ad[i]), ag[i]);
      ad[i] = adi;
      sd.acc(0, r[i], adi);
      sd.acc(1, adi, adi);
    }
    if (!dred<COMP, 2>(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    adad = rd[1];
    ro = __ddiv_rn(rd[0], adad);  // :309
    if (m >= P.nitmax) {          // :313-315 -- last X update, then stop unconverged
      const double nr = -ro;
      for (int i = lo + t; i < hi; i += T) x[i] = add(x[i], mul(nr, d[i]));
      finish(m, m, rmrm, xl, relat);
      return;
    }
  }
}

template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_errmin(Kry2P P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *r = P.r, *ad = P.ad, *atr = P.ag;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  DotAcc<COMP, 2> sd;
  double rd[2];
  int nbar = 0;
  const bool h1 = false;
  double a1 = 0.0;
  auto finish = [&](int status, int m, double rmrm, double xl, int relat) {
    if (P.dsc)
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = m;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rmrm, xl));
      P.ctl->relat = relat;
    }
  };
  sd.zero();
  for (int i = lo + t; i < hi; i += T) sd.acc(0, b[i], b[i]);
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double xl = rd[0];
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }
  const double tol = mul(xl, mul(P.eps, P.eps));
  // R = A X - B, RMRM = GMGM (:126-132)
  sd.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(x[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double ri = sub(a0, b[i]);
    r[i] = ri;
    sd.acc(0, ri, ri);
  }
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double rmrm = rd[0], gmgm = rmrm;
  if (isnan(rmrm)) { finish(ST_NAN, 0, rmrm, xl, relat); return; }
  if (rmrm < mul(mul(P.eps, P.eps), xl)) { finish(ST_OK, 0, rmrm, xl, relat); return; }
  // D = A^T R, D.D (:161-164)
  double *cur = P.d0, *nxt = P.d1;
  sd.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(r[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.St, [&](int j) { return r[j]; });
    cur[i] = a0;
    sd.acc(0, a0, a0);
  }
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double ro = __ddiv_rn(gmgm, rd[0]);  // :176
  // AD = A D (:170) with the first X and R updates (:182, :194) and RMRM
  sd.zero();
  {
    const double nro = -ro;
    for (int i = lo + t; i < hi; i += T) {
      double a0 = diag_term<TD>(cur[i], da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return cur[j]; });
      ad[i] = a0;
      x[i] = add(x[i], mul(nro, cur[i]));
      const double ri = add(r[i], mul(nro, a0));
      r[i] = ri;
      sd.acc(0, ri, ri);
    }
  }
  for (int m = 1;; ++m) {
    if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    const double gm1 = gmgm;
    rmrm = rd[0];
    gmgm = rmrm;
    if (isnan(rmrm)) { finish(ST_NAN, m, rmrm, xl, relat); return; }
    if (rmrm <= tol) { finish(ST_OK, m, rmrm, xl, relat); return; }  // :204
    // A^T R (:232), then every block needs it at neighbours
    for (int i = lo + t; i < hi; i += T) {
      double a0 = diag_term<TD>(r[i], da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.St, [&](int j) { return r[j]; });
      atr[i] = a0;
    }
    if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
    const double beta = __ddiv_rn(gmgm, gm1);  // :235
    // D = BETA D + A^T R (:237-240) where needed, AD = A D (:246), D.D (:252)
    auto dnew = [&](int j) { return add(mul(beta, cur[j]), atr[j]); };
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      const double di = dnew(i);
      double a0 = diag_term<TD>(di, da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, dnew);
      nxt[i] = di;
      ad[i] = a0;
      sd.acc(0, di, di);
    }
    if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    ro = __ddiv_rn(gmgm, rd[0]);  // :253
    { double *tmp = cur; cur = nxt; nxt = tmp; }
    // X = X - RO D (:257), and for the next iteration R = R - RO AD, RMRM
    const double nro = -ro;
    if (m >= P.nitmax) {  // :259
      for (int i = lo + t; i < hi; i += T) x[i] = add(x[i], mul(nro, cur[i]));
      finish(m, m, rmrm, xl, relat);
      return;
    }
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      x[i] = add(x[i], mul(nro, cur[i]));
      const double ri = add(r[i], mul(nro, ad[i]));
      r[i] = ri;
      sd.acc(0, ri, ri);
    }
  }
}

// ---------------------------------------------------------------------------
// CGSQUA (cgsqua.f:151-282, conjugate gradient squared) as ONE persistent
// kernel: per iteration H = A P with K.G0 and H.G0; then H+K (recomputed at
// every node that reads it), X, A(H+K), G with G.G and G.G0; then the local
// P and K updates and a plain grid barrier before the next gather.  GMG0 of
// an iteration is the previous G.G0 (G does not change in between), and
// G.G at the start (G0 = G).
// ---------------------------------------------------------------------------
struct SquaP {
  int npoin, nitmax;
  double eps;
  Sell S;
  const double *da, *dsc;
  double *x;
  const double *b;
  double *g, *g0, *p, *k, *h, *hk;
  double *part;
  Ctl *ctl;
  long long timeout_ns;
};

template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_cgsqua(SquaP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *g = P.g, *g0 = P.g0, *pp = P.p, *kk = P.k, *h = P.h, *hk = P.hk;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  DotAcc<COMP, 2> sd;
  double rd[2];
  int nbar = 0;
  const bool h1 = false;
  double a1 = 0.0;
  auto finish = [&](int status, int m, double rl, double xl, int relat) {
    if (P.dsc)
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = m;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rl, xl));
      P.ctl->relat = relat;
    }
  };
  sd.zero();
  for (int i = lo + t; i < hi; i += T) sd.acc(0, b[i], b[i]);
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double xl = rd[0];
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }
  const double tol = mul(mul(P.eps, P.eps), xl);
  // G = A X - B; G0 = P = K = G (:164-190)
  sd.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(x[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double gi = sub(a0, b[i]);
    g[i] = gi;
    g0[i] = gi;
    pp[i] = gi;
    kk[i] = gi;
    sd.acc(0, gi, gi);
  }
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double rl = rd[0];
  if (isnan(rl)) { finish(ST_NAN, 0, rl, xl, relat); return; }
  if (rl < tol) { finish(ST_OK, 0, rl, xl, relat); return; }  // :172
  double gmg0 = rl;
  for (int m = 1;; ++m) {
    // H = A P (:197), K.G0 and H.G0 (:201)
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      double a0 = diag_term<TD>(pp[i], da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return pp[j]; });
      h[i] = a0;
      const double gi0 = g0[i];
      sd.acc(0, kk[i], gi0);
      sd.acc(1, a0, gi0);
    }
    if (!dred<COMP, 2>(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    const double nro = -__ddiv_rn(rd[0], rd[1]);
    // H+K = -RO H + 2 K (:205-206), X (:211), A(H+K) (:215), G (:224),
    // G.G (:226) and G.G0 (:258)
    auto hpk = [&](int j) { return add(mul(nro, h[j]), mul(2.0, kk[j])); };
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      const double hki = hpk(i);
      double a0 = diag_term<TD>(hki, da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, hpk);
      hk[i] = hki;
      x[i] = add(x[i], mul(nro, hki));
      const double gi = add(g[i], mul(nro, a0));
      g[i] = gi;
      sd.acc(0, gi, gi);
      sd.acc(1, gi, g0[i]);
    }
    if (!dred<COMP, 2>(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    rl = rd[0];
    if (isnan(rl)) { finish(ST_NAN, m, rl, xl, relat); return; }
    if (!(rl > tol)) { finish(ST_OK, m, rl, xl, relat); return; }  // :227
    if (m >= P.nitmax) { finish(m, m, rl, xl, relat); return; }     // :228
    const double beta = __ddiv_rn(rd[1], gmg0);                      // :262
    gmg0 = rd[1];
    const double b2 = mul(beta, beta), tb = mul(2.0, beta);
    // H = H - K; P = BETA**2 P + G + 2 BETA H; K = G + BETA H (:267-280)
    for (int i = lo + t; i < hi; i += T) {
      const double hh = sub(hk[i], kk[i]);
      const double gi = g[i];
      pp[i] = add(add(mul(b2, pp[i]), gi), mul(tb, hh));
      kk[i] = add(gi, mul(beta, hh));
    }
    if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
  }
}

// ---------------------------------------------------------------------------
// CGSTAB (cgstab.f:95-200, BiCGSTAB) without Crout preconditioning, as ONE
// persistent kernel with three grid reductions per iteration: (P.V);
// (T.S, T.T); (R.R, R.P) -- the last pair gives the convergence test and
// the next BETA1.  The new Q, and S, are recomputed at every node that
// reads them (owner's bits); Q and V are double-buffered because the pass
// that writes the new ones reads the old ones at neighbours.
// ---------------------------------------------------------------------------
struct StabP {
  int npoin, nitmax;
  double eps;
  Sell S;
  const double *da, *dsc;
  double *x;
  const double *b;
  double *r, *p, *q0, *q1, *v0, *v1, *s, *t;
  double *part;
  Ctl *ctl;
  long long timeout_ns;
};

template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_cgstab(StabP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *r = P.r, *p = P.p, *sv = P.s, *tv = P.t;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  DotAcc<COMP, 2> sd;
  double rd[2];
  int nbar = 0;
  const bool h1 = false;
  double a1 = 0.0;

  auto finish = [&](int status, int m, double rmrm, double xl, int relat) {
    if (P.dsc)  // solve.f:637-641: X = X*D
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = m;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rmrm, xl));
      P.ctl->relat = relat;
    }
  };

  // XL (:105-111); SQRT(XL) < RMIN: X = 0 (:112-116)
  sd.zero();
  for (int i = lo + t; i < hi; i += T) sd.acc(0, b[i], b[i]);
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double xl = rd[0];
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }
  if (__dsqrt_rn(xl) < 1.0e-15) {
    for (int i = lo + t; i < hi; i += T) x[i] = 0.0;
    finish(ST_OK, 0, 0.0, xl, relat);
    return;
  }
  const double tol = mul(xl, mul(P.eps, P.eps));
  // V = A X, R = B - V, RMRM (:120-123); P = R, V = Q = 0 (:144-147)
  double *qc = P.q0, *qn = P.q1, *vc = P.v0, *vn = P.v1;
  sd.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(x[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double ri = sub(b[i], a0);
    r[i] = ri;
    p[i] = ri;
    qc[i] = 0.0;
    vc[i] = 0.0;
    sd.acc(0, ri, ri);
  }
  if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
  double rmrm = rd[0];
  if (isnan(rmrm)) { finish(ST_NAN, 0, rmrm, xl, relat); return; }
  if (rmrm < mul(mul(P.eps, P.eps), xl)) { finish(ST_OK, 0, rmrm, xl, relat); return; }
  double beta1 = rmrm;  // R.P with P a copy of R: the same products and sum
  double alfa = 1.0, beta = 1.0, omeg1 = 1.0;

  for (int m = 1;; ++m) {
    const double omeg2 = __ddiv_rn(mul(omeg1, beta1), beta);  // :156
    const double omeg = __ddiv_rn(omeg2, alfa);
    beta = beta1;
    const double nomeg2 = -omeg2;
    // Q = R + OMEG Q - OMEG2 V (:161-162), V = A Q (:163), P.V (:173)
    auto qnew = [&](int j) { return add(add(r[j], mul(omeg, qc[j])), mul(nomeg2, vc[j])); };
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      const double qi = qnew(i);
      double a0 = diag_term<TD>(qi, da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, qnew);
      qn[i] = qi;
      vn[i] = a0;
      sd.acc(0, p[i], a0);
    }
    if (!dred_first(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    omeg1 = __ddiv_rn(beta1, rd[0]);  // :174
    { double *tmp = qc; qc = qn; qn = tmp; tmp = vc; vc = vn; vn = tmp; }
    // S = R - OMEG1 V (:176), T = A S (:177), T.S and T.T (:186-187)
    const double nomeg1 = -omeg1;
    auto snew = [&](int j) { return add(r[j], mul(nomeg1, vc[j])); };
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      const double si = snew(i);
      double a0 = diag_term<TD>(si, da, i);
      op_row2<STO>(i, i, h1, a0, a1, P.S, snew);
      sv[i] = si;
      tv[i] = a0;
      sd.acc(0, a0, si);
      sd.acc(1, a0, a0);
    }
    if (!dred<COMP, 2>(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    alfa = __ddiv_rn(rd[0], rd[1]);  // :188
    // X = X + OMEG1 Q + ALFA S (:190-191), R = S - ALFA T (:192), R.R and R.P
    const double nalfa = -alfa;
    sd.zero();
    for (int i = lo + t; i < hi; i += T) {
      x[i] = add(add(x[i], mul(omeg1, qc[i])), mul(alfa, sv[i]));
      const double ri = add(sv[i], mul(nalfa, tv[i]));
      r[i] = ri;
      sd.acc(0, ri, ri);
      sd.acc(1, ri, p[i]);
    }
    if (!dred<COMP, 2>(P.ctl, P.part, P.timeout_ns, nbar, sd, rd)) return;
    rmrm = rd[0];
    beta1 = rd[1];
    if (isnan(rmrm)) { finish(ST_NAN, m, rmrm, xl, relat); return; }
    if (rmrm <= tol) { finish(ST_OK, m, rmrm, xl, relat); return; }  // :194
    if (m >= P.nitmax) { finish(m, m, rmrm, xl, relat); return; }
  }
}

// ---------------------------------------------------------------------------
// GMRES(KRYLOV) (gmres.f:55-213) without preconditioning matrices, as ONE
// persistent kernel.  Columns 1..K-1 by modified Gram-Schmidt: each
// projection's AXPY is fused with the next dot (one grid reduction per
// dot); the normalisation of V(J+1) happens in the pass that computes
// A V(J+1), where every thread that reads V(J+1) at a neighbour scales it
// itself (the owner's bits) and the owner stores it.  Column K: its K+1 dots
// in one pass and one multi-value reduction.  The small dense part (H, the
// Givens rotations, back substitution) is computed by thread 0 of every
// block from identical inputs, so all blocks hold the same scalars.
// ---------------------------------------------------------------------------
constexpr int GM_MAXK = 20;

struct GmP {
  int npoin, nitmax, krylov;
  double eps;
  Sell S;
  const double *da, *dsc;
  double *x;
  const double *b;
  double *r0, *v, *av;   // V(1..K), AV(1..K): K vectors of npoin each
  double *part;          // grid_reduce partials: 8 * G doubles
  double *part_n;        // grid_reduce_n(_comp) partials: 4 * G * (GM_MAXK + 1) doubles
  Ctl *ctl;
  long long timeout_ns;
};

// Reduction of n <= GM_MAXK+1 binary64 values per thread (blocked order of
// each value, as grid_reduce).  vals/out may alias.
static __device__ __noinline__ bool grid_reduce_n(Ctl *ctl, double *part, long long timeout_ns,
                                           int &nbar, const double *vals, int n, double *out) {
  __shared__ double smd[32];
  __shared__ double red_sm[GM_MAXK + 1];
  __shared__ int s_err;
  const int G = gridDim.x, T = blockDim.x, t = threadIdx.x;
  const unsigned long long k = (unsigned long long)(++nbar);
  double *buf = part + (size_t)(k & 1) * (size_t)G * (GM_MAXK + 1);
  for (int q = 0; q < n; ++q) {
    const double bd = block_tree(vals[q], smd);
    if (t == 0) buf[(size_t)blockIdx.x * (GM_MAXK + 1) + q] = bd;
  }
  if (t == 0) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> cnt(ctl->arrivals);
    cnt.fetch_add(1ull, cuda::memory_order_release);
    const unsigned long long target = k * (unsigned long long)G;
    const unsigned long long t0 = global_ns();
    s_err = 0;
    while (cnt.load(cuda::memory_order_acquire) < target) {
      if ((long long)(global_ns() - t0) > timeout_ns) {
        s_err = 1;
        atomicExch(&ctl->status, (int)ST_TIMEOUT);
        break;
      }
      if (SPIN_NS > 0) __nanosleep(SPIN_NS);
    }
  }
  __syncthreads();
  if (s_err) return false;
  for (int q = 0; q < n; ++q) {
    double acc = 0.0;
    for (int bb = t; bb < G; bb += T) acc = add(acc, __ldcg(buf + (size_t)bb * (GM_MAXK + 1) + q));
    const double tot = block_tree(acc, smd);
    if (t == 0) red_sm[q] = tot;
  }
  __syncthreads();
  for (int q = 0; q < n; ++q) out[q] = red_sm[q];
  __syncthreads();
  return true;
}

// The same for compensated values (MODASS = 3): each of the n pairs merged
// as grid_reduce_comp merges one; `part` holds 2 halves of
// G * (GM_MAXK + 1) pairs.  out receives p + s of each.
static __device__ __noinline__ bool grid_reduce_n_comp(Ctl *ctl, double *part,
                                                long long timeout_ns, int &nbar,
                                                const CPair *vals, int n, double *out) {
  __shared__ CPair smc[32];
  __shared__ double red_sm[GM_MAXK + 1];
  __shared__ int s_err;
  const int G = gridDim.x, T = blockDim.x, t = threadIdx.x;
  const unsigned long long k = (unsigned long long)(++nbar);
  double *buf = part + (size_t)(k & 1) * (size_t)G * (GM_MAXK + 1) * 2;
  for (int q = 0; q < n; ++q) {
    const CPair bp = block_tree_c(vals[q], smc);
    if (t == 0) {
      buf[((size_t)blockIdx.x * (GM_MAXK + 1) + q) * 2] = bp.p;
      buf[((size_t)blockIdx.x * (GM_MAXK + 1) + q) * 2 + 1] = bp.s;
    }
  }
  if (t == 0) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> cnt(ctl->arrivals);
    cnt.fetch_add(1ull, cuda::memory_order_release);
    const unsigned long long target = k * (unsigned long long)G;
    const unsigned long long t0 = global_ns();
    s_err = 0;
    while (cnt.load(cuda::memory_order_acquire) < target) {
      if ((long long)(global_ns() - t0) > timeout_ns) {
        s_err = 1;
        atomicExch(&ctl->status, (int)ST_TIMEOUT);
        break;
      }
      if (SPIN_NS > 0) __nanosleep(SPIN_NS);
    }
  }
  __syncthreads();
  if (s_err) return false;
  for (int q = 0; q < n; ++q) {
    CPair acc{0.0, 0.0};
    for (int bb = t; bb < G; bb += T)
      acc = cmerge(acc, CPair{__ldcg(buf + ((size_t)bb * (GM_MAXK + 1) + q) * 2),
                              __ldcg(buf + ((size_t)bb * (GM_MAXK + 1) + q) * 2 + 1)});
    const CPair tot = block_tree_c(acc, smc);
    if (t == 0) red_sm[q] = add(tot.p, tot.s);
  }
  __syncthreads();
  for (int q = 0; q < n; ++q) out[q] = red_sm[q];
  __syncthreads();
  return true;
}

template <int TD, int STO, bool COMP, int MINB = CG_MIN_BLOCKS>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_gmres(GmP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  const size_t N = (size_t)P.npoin;
  double *x = P.x, *r0 = P.r0;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  __shared__ double H[GM_MAXK + 1][GM_MAXK];
  __shared__ double Cg[GM_MAXK], Sg[GM_MAXK], E[GM_MAXK + 1];
  __shared__ int s_flag;
  double vals[GM_MAXK + 1];
  CPair cvals[COMP ? GM_MAXK + 1 : 1];
  DotAcc<COMP, 1> s;
  double red;
  int nbar = 0;
  const bool h1 = false;
  double a1 = 0.0;
  auto V = [&](int j) { return P.v + (size_t)(j - 1) * N; };    // 1-based columns
  auto AV = [&](int j) { return P.av + (size_t)(j - 1) * N; };

  int m = 0, relat = 1;
  double prec = 0.0;
  auto finish = [&]() {
    if (P.dsc)  // solve.f:637-641: X = X*D
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, m < P.nitmax ? ST_OK : m);   // gmres.f:199-214 end messages
      P.ctl->nit = m;
      P.ctl->relres = prec;
      P.ctl->relat = relat;
    }
  };

  // NB = SQRT(B.B), absolute mode below 1 (:67-73)
  s.zero();
  for (int i = lo + t; i < hi; i += T) s.acc(0, b[i], b[i]);
  if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
  double nbn = __dsqrt_rn(red);
  if (nbn < 1.0) { nbn = 1.0; relat = 0; }
  // R0 = A X - B, NR0 (:77-86)
  s.zero();
  for (int i = lo + t; i < hi; i += T) {
    double a0 = diag_term<TD>(x[i], da, i);
    op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int j) { return x[j]; });
    const double r = sub(a0, b[i]);
    r0[i] = r;
    s.acc(0, r, r);
  }
  if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
  double nr0 = __dsqrt_rn(red);
  prec = __ddiv_rn(nr0, nbn);
  if (isnan(prec)) { if (lead) set_status(P.ctl, ST_NAN); return; }
  if (prec <= P.eps) { finish(); return; }   // :87

  for (;;) {
    ++m;                                      // :91
    int K = P.krylov;
    const double c0 = __ddiv_rn(-1.0, nr0);   // :95 V(1) = (-1/NR0) R0
    // The vector V(j) as read at node q: V(1) = c0*R0, V(j>1) = cs*Vraw(j)
    // when its normalisation is pending (cs != 0), else the stored value.
    auto vread = [&](int j, double cs, int q) -> double {
      return j == 1 ? mul(c0, r0[q]) : (cs != 0.0 ? mul(cs, V(j)[q]) : V(j)[q]);
    };
    double cs = 0.0;   // pending scale of the newest column
    for (int J = 1; J <= K - 1; ++J) {
      // AV(J) = A V(J) [storing V(J) normalised]; V(J+1) = AV(J);
      // first MGS dot H(1,J) = V(J+1).V(1)
      double *vj = V(J), *avj = AV(J), *vn = V(J + 1);
      s.zero();
      for (int i = lo + t; i < hi; i += T) {
        const double vi = vread(J, cs, i);
        double a0 = diag_term<TD>(vi, da, i);
        op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int q) { return vread(J, cs, q); });
        avj[i] = a0;
        vn[i] = a0;
        if (J == 1) vj[i] = vi;   // nobody reads V(1) from memory in this pass
        const double v1 = J == 1 ? vi : V(1)[i];
        s.acc(0, a0, v1);
      }
      if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red)) return;
      // every block has finished reading the unscaled V(J): store it scaled
      if (J > 1 && cs != 0.0)
        for (int i = lo + t; i < hi; i += T) vj[i] = mul(cs, vj[i]);
      if (t == 0) H[0][J - 1] = red;
      double hprev = red;
      // I = 2..J: V(J+1) -= H(I-1,J) V(I-1); H(I,J) = V(J+1).V(I)
      for (int I = 2; I <= J + 1; ++I) {
        const double ch = -hprev;
        const double *vp = V(I - 1);
        s.zero();
        for (int i = lo + t; i < hi; i += T) {
          const double u = add(vn[i], mul(ch, vp[i]));
          vn[i] = u;
          const double w = I <= J ? V(I)[i] : u;   // I = J+1: the norm of V(J+1)
          s.acc(0, u, w);
        }
        if (!dred<COMP, 1>(P.ctl, P.part, P.timeout_ns, nbar, s, &red))
          return;
        if (I <= J) {
          if (t == 0) H[I - 1][J - 1] = red;
          hprev = red;
        } else {
          hprev = __dsqrt_rn(red);                // H(J+1,J)
          if (t == 0) H[J][J - 1] = hprev;
        }
      }
      if (hprev < 1.0e-20) {                       // :107-130
        K = J;
        cs = 0.0;
        break;
      }
      cs = __ddiv_rn(1.0, hprev);                 // :131 V(J+1) = V(J+1)/H(J+1,J), deferred
    }
    // AV(K) = A V(K) (:145-151); H(K+1,K) = AV.AV - sum H(I,K)**2 with
    // H(I,K) = AV(K).V(I) (:153-158)
    {
      double *vk = V(K), *avk = AV(K);
      for (int q = 0; q <= K; ++q) {
        if (COMP)
          cvals[q] = CPair{0.0, 0.0};
        else
          vals[q] = 0.0;
      }
      for (int i = lo + t; i < hi; i += T) {
        const double vi = vread(K, cs, i);
        double a0 = diag_term<TD>(vi, da, i);
        op_row2<STO>(i, i, h1, a0, a1, P.S, [&](int q) { return vread(K, cs, q); });
        avk[i] = a0;
        if (COMP)
          cdot_add(cvals[K], a0, a0);
        else
          vals[K] = add(vals[K], mul(a0, a0));
        for (int I = 1; I <= K; ++I) {
          const double vI = I == K ? vi : (I == 1 ? mul(c0, r0[i]) : V(I)[i]);
          if (COMP)
            cdot_add(cvals[I - 1], a0, vI);
          else
            vals[I - 1] = add(vals[I - 1], mul(a0, vI));
        }
      }
      if (COMP) {
        if (!grid_reduce_n_comp(P.ctl, P.part_n, P.timeout_ns, nbar, cvals, K + 1, vals)) return;
      } else if (!grid_reduce_n(P.ctl, P.part_n, P.timeout_ns, nbar, vals, K + 1, vals)) {
        return;
      }
      // all reads of the unscaled V(K) are done: store it as used
      for (int i = lo + t; i < hi; i += T) vk[i] = vread(K, cs, i);
    }
    if (t == 0) {
      double hk = vals[K];
      for (int I = 1; I <= K; ++I) {
        H[I - 1][K - 1] = vals[I - 1];
        hk = sub(hk, mul(vals[I - 1], vals[I - 1]));
      }
      H[K][K - 1] = __dsqrt_rn(hk > 0.0 ? hk : 0.0);
      // Givens rotations (:160-183)
      E[0] = nr0;
      int fail = 0;
      for (int I = 1; I <= K && !fail; ++I) {
        for (int J = 1; J <= I - 1; ++J) {
          const double zz = add(mul(Cg[J - 1], H[J - 1][I - 1]), mul(Sg[J - 1], H[J][I - 1]));
          H[J][I - 1] = add(mul(-Sg[J - 1], H[J - 1][I - 1]), mul(Cg[J - 1], H[J][I - 1]));
          H[J - 1][I - 1] = zz;
        }
        const double rr = __dsqrt_rn(add(mul(H[I - 1][I - 1], H[I - 1][I - 1]),
                                         mul(H[I][I - 1], H[I][I - 1])));
        if (fabs(rr) < 1.0e-6) { fail = 1; break; }
        Cg[I - 1] = __ddiv_rn(H[I - 1][I - 1], rr);
        Sg[I - 1] = __ddiv_rn(H[I][I - 1], rr);
        H[I - 1][I - 1] = rr;
        E[I] = mul(-Sg[I - 1], E[I - 1]);
        E[I - 1] = mul(Cg[I - 1], E[I - 1]);
      }
      if (!fail) {  // back substitution (:184-190)
        E[K - 1] = __ddiv_rn(E[K - 1], H[K - 1][K - 1]);
        for (int J = K - 1; J >= 1; --J) {
          for (int L = J + 1; L <= K; ++L) E[J - 1] = sub(E[J - 1], mul(H[J - 1][L - 1], E[L - 1]));
          E[J - 1] = __ddiv_rn(E[J - 1], H[J - 1][J - 1]);
        }
      }
      s_flag = fail;
    }
    __syncthreads();
    if (s_flag) { finish(); return; }   // R < 1e-6: the solve ends without this update
    // X = X + E(L) V(L), R0 = R0 + E(L) AV(L), L = 1..K (:191-194)
    for (int i = lo + t; i < hi; i += T) {
      double xi = x[i], ri = r0[i];
      for (int L = 1; L <= K; ++L) {
        xi = add(xi, mul(E[L - 1], V(L)[i]));
        ri = add(ri, mul(E[L - 1], AV(L)[i]));
      }
      x[i] = xi;
      r0[i] = ri;
    }
    nr0 = fabs(E[K]);                 // :195
    prec = __ddiv_rn(nr0, nbn);
    if (!(prec >= P.eps && m < P.nitmax)) { finish(); return; }   // :197
    // the next restart reads R0 at neighbours
    if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
  }
}

// ---------------------------------------------------------------------------
// Mixed precision, one launch: a binary32 CG on the binary32 edge-assembled
// copy of the scaled operator (binary32 vectors, products and dot
// accumulation) whose correction z is folded into the binary64 solution
// whenever the recursive binary32 residual has dropped by inner_tol against
// the last true residual (or looks converged).  Each such update
// recomputes the true residual b - A x in binary64 with the binary64
// operator, tests it against outer_tol and restarts the binary32 residual
// from it while keeping the search direction (beta from the recursive
// residual).
// ---------------------------------------------------------------------------
struct MixP {
  int npoin, max_outer, max_inner;
  double outer_tol, inner_tol;
  Sell S;                 // binary64 records + binary32 segments
  const double *da;
  const double *dsc;
  double *x;
  const double *b;
  float *z, *ri, *p0, *p1, *q;
  double *part;
  Ctl *ctl;
  long long timeout_ns;
};

// C16: the binary32 slots' neighbours as 16-bit offsets (EBE meshes whose
// numbering allows it).
template <int TD, int STO, int MINB = CG_MIN_BLOCKS, bool C16 = false>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_mixed(MixP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x;
  const double *b = P.b;
  float *z = P.z, *ri = P.ri, *q = P.q;
  const bool lead = (blockIdx.x == 0 && t == 0);
  double s, red;
  float sf;
  int inner = 0, outer = 0, nbar = 0;

  auto finish = [&](int status, double rr, double xl) {
    if (P.dsc)
      for (int i = lo + t; i < hi; i += T) x[i] = mul(x[i], P.dsc[i]);
    if (lead) {
      set_status(P.ctl, status);
      P.ctl->nit = inner;
      P.ctl->outer = outer;
      P.ctl->relres = __dsqrt_rn(__ddiv_rn(rr, xl));
    }
  };

  s = 0.0;
  for (int i = lo + t; i < hi; i += T) s = add(s, mul(b[i], b[i]));
  if (!grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &red, nullptr)) return;
  double xl = red;
  if (__dsqrt_rn(xl) < 1.0e-15) {
    for (int i = lo + t; i < hi; i += T) x[i] = 0.0;
    finish(ST_OK, 0.0, 1.0);
    return;
  }
  if (xl < 1.0) xl = 1.0;
  const double otol = mul(xl, mul(P.outer_tol, P.outer_tol));
  const float itol2 = (float)mul(P.inner_tol, P.inner_tol);

  // true residual r = b - A x (binary64), r32 = (float)r; rr and rho receive
  // ||r||^2 and ||r32||^2; false on a barrier timeout.
  double rr;
  float rho;
  auto true_residual = [&]() -> bool {
    double sd = 0.0;
    float s32 = 0.0f;
    for (int i = lo + t; i < hi; i += ROW_ILP * T) {
      const int i1 = i + T;
      const bool h1 = ROW_ILP == 2 && i1 < hi;
      double a0 = diag_term<TD>(x[i], P.da, i), a1 = h1 ? diag_term<TD>(x[i1], P.da, i1) : 0.0;
      op_row2<STO>(i, i1, h1, a0, a1, P.S, [&](int j) { return x[j]; });
      const double r0 = sub(b[i], a0);
      sd = add(sd, mul(r0, r0));
      const float q0 = (float)r0;
      ri[i] = q0;
      s32 = add(s32, mul(q0, q0));
      if (h1) {
        const double r1 = sub(b[i1], a1);
        sd = add(sd, mul(r1, r1));
        const float q1 = (float)r1;
        ri[i1] = q1;
        s32 = add(s32, mul(q1, q1));
      }
    }
    return grid_reduce<1, 1>(P.ctl, P.part, P.timeout_ns, nbar, &sd, &s32, &rr, &rho);
  };

  if (!true_residual()) return;
  if (isnan(rr)) { finish(ST_NAN, rr, xl); return; }
  if (rr <= otol) { finish(ST_OK, rr, xl); return; }
  float rmax = rho, beta = 0.0f;
  for (int i = lo + t; i < hi; i += T) z[i] = 0.0f;
  float *cur = P.p0, *nxt = P.p1;
  bool first = true;
  for (;;) {
    // p = r + beta p, evaluated where needed; q = A32 p; p.q
    sf = 0.0f;
    for (int i = lo + t; i < hi; i += ROW_ILP * T) {
      const int i1 = i + T;
      const bool h1 = ROW_ILP == 2 && i1 < hi;
      float p0, p1 = 0.0f, a0, a1;
      if (first) {
        p0 = ri[i];
        if (h1) p1 = ri[i1];
        seg_row2<C16>(i, i1, h1, p0, p1, a0, a1, P.S, [&](int k) { return ri[k]; });
      } else {
        p0 = add(ri[i], mul(beta, cur[i]));
        if (h1) p1 = add(ri[i1], mul(beta, cur[i1]));
        seg_row2<C16>(i, i1, h1, p0, p1, a0, a1, P.S,
                      [&](int k) { return add(ri[k], mul(beta, cur[k])); });
      }
      nxt[i] = p0;
      q[i] = a0;
      sf = add(sf, mul(p0, a0));
      if (h1) {
        nxt[i1] = p1;
        q[i1] = a1;
        sf = add(sf, mul(p1, a1));
      }
    }
    float pq;
    if (!grid_reduce<0, 1>(P.ctl, P.part, P.timeout_ns, nbar, nullptr, &sf, nullptr, &pq)) return;
    if (!(pq > 0.0f)) { finish(isnan(pq) ? ST_NAN : ST_BREAKDOWN, rr, xl); return; }
    const float alpha = __fdiv_rn(rho, pq);
    sf = 0.0f;
    for (int i = lo + t; i < hi; i += T) {
      z[i] = add(z[i], mul(alpha, nxt[i]));
      const float rv = sub(ri[i], mul(alpha, q[i]));
      ri[i] = rv;
      sf = add(sf, mul(rv, rv));
    }
    float rho_new;
    if (!grid_reduce<0, 1>(P.ctl, P.part, P.timeout_ns, nbar, nullptr, &sf, nullptr, &rho_new)) return;
    const float rho_rec = rho_new, rho_old = rho;
    ++inner;
    { float *tmp = cur; cur = nxt; nxt = tmp; }
    const bool last = inner >= P.max_inner;
    if (last || rho_new <= mul(itol2, rmax) || (double)rho_new <= otol) {
      // reliable update: x += z in binary64, then the true residual
      for (int i = lo + t; i < hi; i += T) {
        x[i] = add(x[i], (double)z[i]);
        z[i] = 0.0f;
      }
      if (!grid_sync(P.ctl, P.part, P.timeout_ns, nbar)) return;
      if (!true_residual()) return;
      ++outer;
      if (isnan(rr)) { finish(ST_NAN, rr, xl); return; }
      if (rr <= otol) { finish(ST_OK, rr, xl); return; }
      if (last || outer >= P.max_outer) { finish(inner, rr, xl); return; }
      rho_new = rho;
      rmax = rho;
    }
    beta = __fdiv_rn(rho_rec, rho_old);
    rho = rho_new;
    first = false;
  }
}

// ---------------------------------------------------------------------------
// Wave-equation operator assembly (mt01aa.f, mt02aa.f:106-149, ASSVEC
// diagonals, OM 'M=M+N').  Element pass writes XM and the element diagonal
// terms; node pass sums the diagonals in ASSVEC order.
// ew layout: [0] mass diagonal (same for the three points), [1..3] diffusion
// diagonal of points 1..3.
// ---------------------------------------------------------------------------
__global__ void k_wave_elems(int nelem, const int *__restrict__ ik, const double *__restrict__ xc,
                             const double *__restrict__ yc, const double *__restrict__ coef,
                             double *xm, double *ew, int *err) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    const int i1 = ik[e], i2 = ik[(size_t)nelem + e], i3 = ik[2 * (size_t)nelem + e];
    const double x1 = xc[i1], y1 = yc[i1];
    const double X2 = sub(xc[i2], x1), X3 = sub(xc[i3], x1);  // inbief.f:385-391
    const double Y2 = sub(yc[i2], y1), Y3 = sub(yc[i3], y1);
    const double surf = mul(0.5, sub(mul(X2, Y3), mul(X3, Y2)));  // surv11.f:63
    if (sub(mul(X2, Y3), mul(Y2, X3)) < 1.0e-20) atomicExch(err, 1);  // geoelt.f:82
    // MT01AA, XMUL = 1
    const double det = mul(surf, __ddiv_rn(1.0, 12.0));
    // MT02AA, P0 isotropic, XMUL = 1, U = coef
    const double s2d = __ddiv_rn(mul(1.0, 0.25), surf);
    const double visc1 = mul(coef[e], s2d);
    const double bpe = mul(visc1, add(mul(Y3, Y3), mul(X3, X3)));
    const double cpf = mul(visc1, add(mul(Y2, Y3), mul(X2, X3)));
    const double apd = mul(visc1, add(mul(Y2, Y2), mul(X2, X2)));
    // OM 'M=M+N': XM(mass) + XM(diffusion)
    xm[e] = add(det, sub(cpf, bpe));
    xm[(size_t)nelem + e] = add(det, sub(cpf, apd));
    xm[2 * (size_t)nelem + e] = add(det, -cpf);
    ew[e] = add(det, det);
    ew[(size_t)nelem + e] = sub(add(apd, bpe), mul(2.0, cpf));
    ew[2 * (size_t)nelem + e] = bpe;
    ew[3 * (size_t)nelem + e] = apd;
  }
}

// AM1 = MT01AA(xmul_mass) 'M=N' then 'M=M+N' with MT02AA(xmul_dif), the
// general form of PROPAG's wave-equation operator (propag.F:673-676,
// 1407-1408).  KIND 10: MATDIF, U per element (mt02aa.f:106-149); 11:
// MATDIF, U per node (mt02aa.f:244-279); 12: MATDIFUV, U and V per node
// (mt02aa.f:200-240).  Same output layout as k_wave_elems (XM summed, the
// element diagonals of each matrix kept apart for their ASSVEC sums).
template <int KIND>
__global__ void k_mass_diff_elems(int nelem, const int *__restrict__ ik,
                                  const double *__restrict__ xc, const double *__restrict__ yc,
                                  double xmul_mass, double xmul_dif,
                                  const double *__restrict__ u, const double *__restrict__ v,
                                  double *xm, double *ew, int *err) {
  const double sur12 = __ddiv_rn(xmul_mass, 12.0);  // mt01aa.f:83
  const double xsur12 = __ddiv_rn(xmul_dif, 12.0);  // mt02aa.f:97
  const double xsur48 = __ddiv_rn(xmul_dif, 48.0);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    const int i1 = ik[e], i2 = ik[(size_t)nelem + e], i3 = ik[2 * (size_t)nelem + e];
    const double x1 = xc[i1], y1 = yc[i1];
    const double X2 = sub(xc[i2], x1), X3 = sub(xc[i3], x1);  // inbief.f:385-391
    const double Y2 = sub(yc[i2], y1), Y3 = sub(yc[i3], y1);
    const double surf = mul(0.5, sub(mul(X2, Y3), mul(X3, Y2)));  // surv11.f:63
    if (sub(mul(X2, Y3), mul(Y2, X3)) < 1.0e-20) atomicExch(err, 1);  // geoelt.f:82
    const double det = mul(surf, sur12);  // mt01aa.f:91
    double a11, a22, a33, a12, a13, a23;
    if (KIND == 10) {
      const double s2d = __ddiv_rn(mul(xmul_dif, 0.25), surf);
      const double visc1 = mul(u[e], s2d);
      const double bpe = mul(visc1, add(mul(Y3, Y3), mul(X3, X3)));
      const double cpf = mul(visc1, add(mul(Y2, Y3), mul(X2, X3)));
      const double apd = mul(visc1, add(mul(Y2, Y2), mul(X2, X2)));
      a11 = sub(add(apd, bpe), mul(2.0, cpf));
      a22 = bpe;
      a33 = apd;
      a12 = sub(cpf, bpe);
      a13 = sub(cpf, apd);
      a23 = -cpf;
    } else {
      if (KIND == 11) {
        const double somvx = __ddiv_rn(mul(add(add(u[i1], u[i2]), u[i3]), xsur12), surf);
        const double x2x3 = add(mul(X2, X3), mul(Y2, Y3));
        const double x2aux = add(mul(X2, add(-X2, X3)), mul(Y2, add(-Y2, Y3)));
        const double x3aux = add(mul(X3, add(-X2, X3)), mul(Y3, add(-Y2, Y3)));
        a12 = -mul(somvx, x3aux);
        a13 = mul(somvx, x2aux);
        a23 = -mul(somvx, x2x3);
      } else {
        const double g1 = v[i1], g2 = v[i2], g3 = v[i3];
        const double coef1 = __ddiv_rn(xsur48, surf);
        const double g123 = add(add(g1, g2), g3);
        const double coef2 = add(add(mul(u[i1], add(g1, g123)), mul(u[i2], add(g2, g123))),
                                 mul(u[i3], add(g3, g123)));
        a12 = mul(mul(add(mul(Y3, sub(Y2, Y3)), mul(X3, sub(X2, X3))), coef2), coef1);
        a13 = -mul(mul(add(mul(Y2, sub(Y2, Y3)), mul(X2, sub(X2, X3))), coef2), coef1);
        a23 = -mul(mul(add(mul(Y2, Y3), mul(X2, X3)), coef2), coef1);
      }
      a11 = sub(-a12, a13);
      a22 = sub(-a12, a23);
      a33 = sub(-a13, a23);
    }
    // OM 'M=M+N': XM(mass) + XM(diffusion)
    xm[e] = add(det, a12);
    xm[(size_t)nelem + e] = add(det, a13);
    xm[2 * (size_t)nelem + e] = add(det, a23);
    ew[e] = add(det, det);
    ew[(size_t)nelem + e] = a11;
    ew[2 * (size_t)nelem + e] = a22;
    ew[3 * (size_t)nelem + e] = a33;
  }
}

__global__ void k_wave_nodes(int npoin, const int *__restrict__ ptr, const int *__restrict__ ek,
                             int nelem, const double *__restrict__ ew, double *dm) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    double sm = 0.0, sd = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
      const int p = ek[j], e = p >> 2, k = p & 3;
      sm = add(sm, ew[e]);
      sd = add(sd, ew[(size_t)(1 + k) * nelem + e]);
    }
    dm[i] = add(sm, sd);
  }
}

// Per-element gradient g_e = -lambda_e^T K_e x_e with K_e the unit-
// coefficient MT02AA element matrix (rows sum to zero, so
// lambda^T K x = -sum_{k<l} K_kl (lambda_k - lambda_l)(x_k - x_l)).
__global__ void k_coef_grad(int nelem, const int *__restrict__ ik, const double *__restrict__ xc,
                            const double *__restrict__ yc, const double *__restrict__ lam,
                            const double *__restrict__ xs, double *grad) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    const int i1 = ik[e], i2 = ik[(size_t)nelem + e], i3 = ik[2 * (size_t)nelem + e];
    const double x1 = xc[i1], y1 = yc[i1];
    const double X2 = xc[i2] - x1, X3 = xc[i3] - x1;
    const double Y2 = yc[i2] - y1, Y3 = yc[i3] - y1;
    const double surf = 0.5 * (X2 * Y3 - X3 * Y2);
    const double s2d = 0.25 / surf;
    const double bpe = s2d * (Y3 * Y3 + X3 * X3);
    const double cpf = s2d * (Y2 * Y3 + X2 * X3);
    const double apd = s2d * (Y2 * Y2 + X2 * X2);
    const double k12 = cpf - bpe, k13 = cpf - apd, k23 = -cpf;
    const double l1 = lam[i1], l2 = lam[i2], l3 = lam[i3];
    const double u1 = xs[i1], u2 = xs[i2], u3 = xs[i3];
    const double lkx = -(k12 * (l1 - l2) * (u1 - u2) + k13 * (l1 - l3) * (u1 - u3) +
                         k23 * (l2 - l3) * (u2 - u3));
    grad[e] = -lkx;
  }
}

// Adjoint gradients of the node-coefficient diffusion forms (the operators
// of k_mass_diff_elems, KIND 11 and 12).  With A^T lam = dL/dx, an
// element's sensitivity to its scalar factor is s_e = -lam_e^T Ghat_e x_e,
// Ghat_e the element matrix per unit factor (zero row sums, so
// lam^T Ghat x = -sum_{k<l} Ghat_kl (lam_k - lam_l)(x_k - x_l)):
//   KIND 11: factor SOMVX = (U1+U2+U3) XMUL/(12 S), dSOMVX/dU_k = XMUL/(12 S);
//            ew[e] = s_e XMUL/(12 S)
//   KIND 12: factor COEF2 * COEF1, COEF2 = sum_k U_k (V_k + G123),
//            COEF1 = XMUL/(48 S); ew[e] = s_e COEF1, ew[ne+e] = G123 =
//            V1+V2+V3, ew[2ne+e] = U1+U2+U3
// The node pass then sums over the node's elements (no atomics):
//   KIND 11: dL/dU_i = sum_e ew[e]
//   KIND 12: dL/dU_i = sum_e ew[e] (V_i + G123_e),
//            dL/dV_i = sum_e ew[e] (U_i + U1+U2+U3)
template <int KIND>
__global__ void k_mass_diff_grad_elems(int nelem, const int *__restrict__ ik,
                                       const double *__restrict__ xc,
                                       const double *__restrict__ yc, double xmul_dif,
                                       const double *__restrict__ u,
                                       const double *__restrict__ v,
                                       const double *__restrict__ lam,
                                       const double *__restrict__ xs, double *ew) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    const int i1 = ik[e], i2 = ik[(size_t)nelem + e], i3 = ik[2 * (size_t)nelem + e];
    const double x1 = xc[i1], y1 = yc[i1];
    const double X2 = xc[i2] - x1, X3 = xc[i3] - x1;
    const double Y2 = yc[i2] - y1, Y3 = yc[i3] - y1;
    const double surf = 0.5 * (X2 * Y3 - X3 * Y2);
    double g12, g13, g23, scale;
    if (KIND == 11) {
      g12 = -(X3 * (X3 - X2) + Y3 * (Y3 - Y2));
      g13 = X2 * (X3 - X2) + Y2 * (Y3 - Y2);
      g23 = -(X2 * X3 + Y2 * Y3);
      scale = xmul_dif / 12.0 / surf;
    } else {
      g12 = Y3 * (Y2 - Y3) + X3 * (X2 - X3);
      g13 = -(Y2 * (Y2 - Y3) + X2 * (X2 - X3));
      g23 = -(Y2 * Y3 + X2 * X3);
      scale = xmul_dif / 48.0 / surf;
    }
    const double l1 = lam[i1], l2 = lam[i2], l3 = lam[i3];
    const double w1 = xs[i1], w2 = xs[i2], w3 = xs[i3];
    const double lgx = -(g12 * (l1 - l2) * (w1 - w2) + g13 * (l1 - l3) * (w1 - w3) +
                         g23 * (l2 - l3) * (w2 - w3));
    ew[e] = -lgx * scale;
    if (KIND == 12) {
      ew[(size_t)nelem + e] = v[i1] + v[i2] + v[i3];
      ew[2 * (size_t)nelem + e] = u[i1] + u[i2] + u[i3];
    }
  }
}

template <int KIND>
__global__ void k_mass_diff_grad_nodes(int npoin, const int *__restrict__ ptr,
                                       const int *__restrict__ ek, int nelem,
                                       const double *__restrict__ ew,
                                       const double *__restrict__ u,
                                       const double *__restrict__ v, double *gu, double *gv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    double su = 0.0, sv = 0.0;
    const double ui = KIND == 12 ? u[i] : 0.0, vi = KIND == 12 ? v[i] : 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
      const int e = ek[j] >> 2;
      const double se = ew[e];
      if (KIND == 11) {
        su += se;
      } else {
        su += se * (vi + ew[(size_t)nelem + e]);
        sv += se * (ui + ew[2 * (size_t)nelem + e]);
      }
    }
    gu[i] = su;
    if (KIND == 12) gv[i] = sv;
  }
}

}  // namespace bief
