// bief_batch.cuh -- many independent meshes solved in ONE persistent launch.
//
// The instances are the diagonal blocks of one block-diagonal mesh (each
// instance's nodes a contiguous range starting on a multiple of 32).  Each
// instance runs the mixed-precision algorithm of k_mixed (binary32 CG on the
// edge-assembled difference-form operator, binary64 reliable updates) with
// its own scalars and its own convergence mask; all instances advance in
// lock-step phases separated by grid barriers, and an instance that has
// converged stops taking work.
//
// Work unit: a tile of C = blockDim.x * npt consecutive nodes of one
// instance (thread t: nodes t, t+T, ... of the tile).  After every barrier
// each block rebuilds, in shared memory, the prefix sums of the tile
// counts of the still-active instances and takes active tiles b, b+G, ...
// Per-instance dot products: each tile's block reduces its thread partials
// (block_tree's tree) into a per-tile slot; one warp per instance then adds
// the instance's tile partials (lane l: tiles l, l+32, ...) and folds the
// lanes with a xor-butterfly.  Every block performs these reductions and the
// scalar updates of every instance itself, in the same order, so all blocks
// hold identical copies of the per-instance state without further traffic.
#pragma once

#include "bief_kernels.cuh"

namespace bief {

constexpr int BATCH_MAX_INST = 512;
enum : int { BS_ITER = 0, BS_UPD = 1, BS_DONE = 2 };

struct BatchP {
  int ninst, npt, max_outer, max_inner;
  double outer_tol, inner_tol;
  const int *inst_off;  // [ninst] first node of each instance
  const int *inst_n;    // [ninst] nodes of each instance
  const int *inst_t0;   // [ninst+1] first tile of each instance (prefix)
  Sell S;
  const double *da, *dsc;
  double *x;
  const double *b;
  float *z, *ri, *p0, *p1, *q;
  double *part;         // two halves of 2 * ntiles slots
  int ntiles;
  Ctl *ctl;
  int *st_out, *inner_out, *outer_out;
  double *relres_out;
  long long timeout_ns;
};

// Per-instance state, one copy per block in shared memory.
struct BatchState {
  int state[BATCH_MAX_INST], inner[BATCH_MAX_INST], outer[BATCH_MAX_INST];
  int status[BATCH_MAX_INST], act[BATCH_MAX_INST + 1];
  unsigned char first[BATCH_MAX_INST], par[BATCH_MAX_INST], last[BATCH_MAX_INST];
  float rho[BATCH_MAX_INST], rmax[BATCH_MAX_INST], beta[BATCH_MAX_INST];
  float alpha[BATCH_MAX_INST], rho_rec[BATCH_MAX_INST], rho_old[BATCH_MAX_INST];
  double rr[BATCH_MAX_INST], xl[BATCH_MAX_INST], otol[BATCH_MAX_INST];
};

template <int STO, class V>
__device__ __forceinline__ double op_row(int i, double acc, const Sell &S, V vec) {
  double unused = 0.0;
  op_row2<STO>(i, i, false, acc, unused, S, vec);
  return acc;
}

template <int TD, int STO, int MINB = CG_MIN_BLOCKS, bool C16 = false>
__global__ void __launch_bounds__(CG_THREADS, MINB) k_batch(BatchP P) {
  __shared__ BatchState B;
  const int T = blockDim.x, t = threadIdx.x, G = gridDim.x;
  const int warp = t >> 5, lane = t & 31, nwarps = T >> 5;
  const int C = T * P.npt;
  const int NI = P.ninst;
  int nbar = 0;
  const float itol2 = (float)mul(P.inner_tol, P.inner_tol);

  // prefix sums of the tile counts of the active instances (warp 0: each
  // lane sums a run of consecutive instances, then a warp scan)
  auto rebuild_active = [&]() {
    __syncthreads();
    if (warp == 0) {
      const int per = (NI + 31) / 32, i0 = min(NI, lane * per), i1 = min(NI, i0 + per);
      int a = 0;
      for (int i = i0; i < i1; ++i)
        if (B.state[i] != BS_DONE) a += P.inst_t0[i + 1] - P.inst_t0[i];
      int incl = a;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
      }
      int run = incl - a;
      for (int i = i0; i < i1; ++i) {
        B.act[i] = run;
        if (B.state[i] != BS_DONE) run += P.inst_t0[i + 1] - P.inst_t0[i];
      }
      if (lane == 31) B.act[NI] = incl;
    }
    __syncthreads();
  };
  // active tile a -> instance (binary search on B.act)
  auto inst_of = [&](int a) {
    int lo = 0, hi = NI - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (B.act[mid] <= a) lo = mid; else hi = mid - 1;
    }
    return lo;
  };
  // partials written before barrier k go to half (k-1)&1 (nbar = k-1 while
  // writing, = k while reading), so one phase never overwrites the partials
  // a slower block may still be reading from the previous barrier
  auto half = [&]() { return P.part + (size_t)(nbar & 1) * 2 * P.ntiles; };
  // Tile partials in two stages, the two stages of block_tree: each warp
  // folds its lanes' partials of a tile (xor butterfly) into shared memory
  // as the tile ends; the tiles a block handles in a phase (up to MAXT at a
  // time) are then finished together -- per tile, the warp sums in warp
  // order, zero-padded to 32, through a second butterfly -- after one
  // __syncthreads, instead of two block-wide syncs per tile.  Same tree,
  // same bits.
  constexpr int MAXT = 16;
  __shared__ double W[MAXT][2][32];
  __shared__ int Wgt[MAXT];
  __shared__ unsigned char Wk[MAXT][2];  // 0 none, 1 binary64, 2 binary32
  int ntl = 0;                           // tiles held (uniform in the block)
  if (t < 2 * MAXT) Wk[t >> 1][t & 1] = 0;
  auto flush = [&]() {
    __syncthreads();
    for (int pr = warp; pr < 2 * ntl; pr += nwarps) {
      const int tl = pr >> 1, q = pr & 1, kind = Wk[tl][q];
      if (kind == 0) continue;
      double *dst = half() + 2 * (size_t)Wgt[tl] + q;
      if (kind == 1) {
        double u = lane < nwarps ? W[tl][q][lane] : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) u = add(u, __shfl_xor_sync(0xffffffffu, u, o));
        if (lane == 0) *dst = u;
      } else {
        float u = lane < nwarps ? (float)W[tl][q][lane] : 0.0f;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) u = add(u, __shfl_xor_sync(0xffffffffu, u, o));
        if (lane == 0) *dst = (double)u;
      }
      if (lane == 0) Wk[tl][q] = 0;
    }
    __syncthreads();
    ntl = 0;
  };
  auto store64 = [&](double v, int gt, int q) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = add(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) W[ntl][q][warp] = v;
    if (t == 0) { Wgt[ntl] = gt; Wk[ntl][q] = 1; }
  };
  auto store32 = [&](float v, int gt, int q) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = add(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) W[ntl][q][warp] = (double)v;
    if (t == 0) { Wgt[ntl] = gt; Wk[ntl][q] = 2; }
  };
  // Per-instance sums of the tile partials of the last barrier: one warp
  // per instance, lane l adds the instance's tiles l, l+32, ... left to
  // right, then a xor-butterfly (offsets 16..1) -- four instances of a warp
  // at a time, with their loads interleaved.  need(i): 1 = slot 0 in binary64, 2 = slot 0 in
  // binary32, 4 = slot 1 in binary32 (or-ed).  Results in SA[i] (slot 0)
  // and SB[i] (slot 1), which reuse the tile buffer (idle between phases);
  // valid in the whole block after the closing __syncthreads.
  double *SA = &W[0][0][0], *SB = &W[0][0][0] + BATCH_MAX_INST;
  auto gather_sums = [&](auto need) {
    const double *h = P.part + (size_t)((nbar - 1) & 1) * 2 * P.ntiles;
    for (int i0 = 4 * warp; i0 < NI; i0 += 4 * nwarps) {
      int nd[4], k0[4], k1[4];
      double s64[4];
      float s0[4], s1[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int i = i0 + c;
        nd[c] = i < NI ? need(i) : 0;
        k0[c] = nd[c] ? P.inst_t0[i] + lane : 0;
        k1[c] = nd[c] ? P.inst_t0[i + 1] : 0;
        s64[c] = 0.0;
        s0[c] = 0.0f;
        s1[c] = 0.0f;
      }
      for (;;) {
        bool any = false;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (k0[c] < k1[c]) {
            any = true;
            const double v0 = __ldcg(h + 2 * (size_t)k0[c]);
            if (nd[c] & 1) s64[c] = add(s64[c], v0);
            if (nd[c] & 2) s0[c] = add(s0[c], (float)v0);
            if (nd[c] & 4) s1[c] = add(s1[c], (float)__ldcg(h + 2 * (size_t)k0[c] + 1));
            k0[c] += 32;
          }
        }
        if (!__any_sync(0xffffffffu, any)) break;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
          s64[c] = add(s64[c], __shfl_xor_sync(0xffffffffu, s64[c], o));
          s0[c] = add(s0[c], __shfl_xor_sync(0xffffffffu, s0[c], o));
          s1[c] = add(s1[c], __shfl_xor_sync(0xffffffffu, s1[c], o));
        }
        if (lane == 0 && nd[c]) {
          SA[i0 + c] = (nd[c] & 1) ? s64[c] : (double)s0[c];
          SB[i0 + c] = (double)s1[c];
        }
      }
    }
    __syncthreads();
  };
  // for every active tile handled by this block: body(i, gtile, n0, n1);
  // the tiles' partials are complete in `part` when it returns
  auto for_tiles = [&](auto body) {
    const int A = B.act[NI];
    for (int a = blockIdx.x; a < A; a += G) {
      const int i = inst_of(a);
      const int k = a - B.act[i];
      const int n0 = P.inst_off[i] + k * C;
      const int n1 = P.inst_off[i] + min((k + 1) * C, P.inst_n[i]);
      body(i, P.inst_t0[i] + k, n0, n1);
      if (++ntl == MAXT) flush();
    }
    if (ntl) flush();
  };

  // ---- initial state
  for (int i = t; i < NI; i += T) {
    B.state[i] = BS_ITER;
    B.inner[i] = 0;
    B.outer[i] = 0;
    B.status[i] = ST_OK;
    B.first[i] = 1;
    B.par[i] = 0;
    B.last[i] = 0;
  }
  rebuild_active();

  // ---- phase I0: xl = b.b
  for_tiles([&](int i, int gt, int n0, int n1) {
    double s = 0.0;
    for (int j = 0; j < P.npt; ++j) {
      const int v = n0 + t + j * T;
      if (v < n1) s = add(s, mul(P.b[v], P.b[v]));
    }
    store64(s, gt, 0);
  });
  if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
  gather_sums([&](int i) { return 1; });
  for (int i = t; i < NI; i += T) {
    double xl = SA[i];
    if (__dsqrt_rn(xl) < 1.0e-15) {
      B.state[i] = BS_UPD;   // marker: zero solution in the next phase
      B.last[i] = 2;
      xl = 1.0;
    }
    if (xl < 1.0) xl = 1.0;
    B.xl[i] = xl;
    B.otol[i] = mul(xl, mul(P.outer_tol, P.outer_tol));
  }
  __syncthreads();

  // true residual r = b - A x (binary64 records), r32, rr and rho partials
  auto true_residual = [&](int gt, int n0, int n1, bool zero_z) {
    double sd = 0.0;
    float s32 = 0.0f;
    for (int j = 0; j < P.npt; ++j) {
      const int v = n0 + t + j * T;
      if (v < n1) {
        double acc = diag_term<TD>(P.x[v], P.da, v);
        acc = op_row<STO>(v, acc, P.S, [&](int w) { return P.x[w]; });
        const double rv = sub(P.b[v], acc);
        sd = add(sd, mul(rv, rv));
        const float r32 = (float)rv;
        P.ri[v] = r32;
        s32 = add(s32, mul(r32, r32));
        if (zero_z) P.z[v] = 0.0f;
      }
    }
    store64(sd, gt, 0);
    store32(s32, gt, 1);
  };

  // ---- phase I1: true residual (instances with b = 0: x = 0)
  for_tiles([&](int i, int gt, int n0, int n1) {
    if (B.last[i] == 2) {
      for (int j = 0; j < P.npt; ++j) {
        const int v = n0 + t + j * T;
        if (v < n1) P.x[v] = 0.0;
      }
    } else {
      true_residual(gt, n0, n1, true);
    }
  });
  if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
  gather_sums([&](int i) { return B.last[i] == 2 ? 0 : 1 | 4; });
  for (int i = t; i < NI; i += T) {
    if (B.last[i] == 2) {
      B.state[i] = BS_DONE;
      B.rr[i] = 0.0;
      B.last[i] = 0;
      continue;
    }
    const double rr = SA[i];
    const float rho = (float)SB[i];
    B.rr[i] = rr;
    if (isnan(rr)) { B.state[i] = BS_DONE; B.status[i] = ST_NAN; }
    else if (rr <= B.otol[i]) { B.state[i] = BS_DONE; }
    else { B.rho[i] = rho; B.rmax[i] = rho; B.beta[i] = 0.0f; B.state[i] = BS_ITER; }
  }
  rebuild_active();

  // ---- main loop: two phases per cycle
  while (B.act[NI] > 0) {
    // phase A: ITER -> p, q = A32 p, p.q ; UPD -> x += z, z = 0
    for_tiles([&](int i, int gt, int n0, int n1) {
      if (B.state[i] == BS_ITER) {
        float *cur = B.par[i] ? P.p1 : P.p0, *nxt = B.par[i] ? P.p0 : P.p1;
        const float beta = B.beta[i];
        const bool first = B.first[i];
        float s = 0.0f;
        for (int j = 0; j < P.npt; ++j) {
          const int v = n0 + t + j * T;
          if (v < n1) {
            float pi, acc;
            if (first) {
              pi = P.ri[v];
              acc = seg_row<C16>(v, pi, P.S, [&](int w) { return P.ri[w]; });
            } else {
              pi = add(P.ri[v], mul(beta, cur[v]));
              acc = seg_row<C16>(v, pi, P.S,
                                 [&](int w) { return add(P.ri[w], mul(beta, cur[w])); });
            }
            nxt[v] = pi;
            P.q[v] = acc;
            s = add(s, mul(pi, acc));
          }
        }
        store32(s, gt, 0);
      } else {
        for (int j = 0; j < P.npt; ++j) {
          const int v = n0 + t + j * T;
          if (v < n1) {
            P.x[v] = add(P.x[v], (double)P.z[v]);
            P.z[v] = 0.0f;
          }
        }
      }
    });
    if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
    gather_sums([&](int i) { return B.state[i] == BS_ITER ? 2 : 0; });
    for (int i = t; i < NI; i += T) {
      if (B.state[i] != BS_ITER) continue;
      const float pq = (float)SA[i];
      if (!(pq > 0.0f)) {
        B.state[i] = BS_DONE;
        B.status[i] = isnan(pq) ? ST_NAN : ST_BREAKDOWN;
      } else {
        B.alpha[i] = __fdiv_rn(B.rho[i], pq);
      }
    }
    rebuild_active();

    // phase B: ITER -> z += alpha p, r -= alpha q, r.r ; UPD -> true residual
    for_tiles([&](int i, int gt, int n0, int n1) {
      if (B.state[i] == BS_ITER) {
        float *nxt = B.par[i] ? P.p0 : P.p1;
        const float alpha = B.alpha[i];
        float s = 0.0f;
        for (int j = 0; j < P.npt; ++j) {
          const int v = n0 + t + j * T;
          if (v < n1) {
            P.z[v] = add(P.z[v], mul(alpha, nxt[v]));
            const float rv = sub(P.ri[v], mul(alpha, P.q[v]));
            P.ri[v] = rv;
            s = add(s, mul(rv, rv));
          }
        }
        store32(s, gt, 0);
      } else {
        true_residual(gt, n0, n1, false);
      }
    });
    if (!grid_barrier(P.ctl, P.timeout_ns, nbar)) return;
    gather_sums([&](int i) {
      return B.state[i] == BS_ITER ? 2 : (B.state[i] == BS_UPD ? 1 | 4 : 0);
    });
    for (int i = t; i < NI; i += T) {
      if (B.state[i] == BS_ITER) {
        const float rho_new = (float)SA[i];
        const float rho_old = B.rho[i];
        B.inner[i] += 1;
        B.par[i] ^= 1;
        const bool last = B.inner[i] >= P.max_inner;
        if (last || rho_new <= mul(itol2, B.rmax[i]) || (double)rho_new <= B.otol[i]) {
          B.state[i] = BS_UPD;
          B.rho_rec[i] = rho_new;
          B.rho_old[i] = rho_old;
          B.last[i] = last ? 1 : 0;
        } else {
          B.beta[i] = __fdiv_rn(rho_new, rho_old);
          B.rho[i] = rho_new;
          B.first[i] = 0;
        }
      } else if (B.state[i] == BS_UPD) {
        const double rr = SA[i];
        const float rho = (float)SB[i];
        B.rr[i] = rr;
        B.outer[i] += 1;
        if (isnan(rr)) {
          B.state[i] = BS_DONE;
          B.status[i] = ST_NAN;
        } else if (rr <= B.otol[i]) {
          B.state[i] = BS_DONE;
        } else if (B.last[i] || B.outer[i] >= P.max_outer) {
          B.state[i] = BS_DONE;
          B.status[i] = B.inner[i];
        } else {
          B.rmax[i] = rho;
          B.beta[i] = __fdiv_rn(B.rho_rec[i], B.rho_old[i]);
          B.rho[i] = rho;
          B.first[i] = 0;
          B.state[i] = BS_ITER;
        }
      }
    }
    rebuild_active();
  }

  // ---- undo the change of variables, report
  if (P.dsc) {
    const int n0 = P.inst_off[0];
    const int nlast = P.inst_off[NI - 1] + P.inst_n[NI - 1];
    for (int v = n0 + blockIdx.x * T + t; v < nlast; v += G * T) P.x[v] = mul(P.x[v], P.dsc[v]);
  }
  if (blockIdx.x == 0) {
    for (int i = t; i < NI; i += T) {
      P.st_out[i] = B.status[i];
      P.inner_out[i] = B.inner[i];
      P.outer_out[i] = B.outer[i];
      P.relres_out[i] = __dsqrt_rn(__ddiv_rn(B.rr[i], B.xl[i]));
    }
  }
}

// Every element's three nodes belong to the same instance (binary search
// of the instance ranges); otherwise the batch is not block diagonal (and
// neither is its segment numbering, whose segments are element faces).
__global__ void k_check_blockdiag(int nelem, const int *__restrict__ ik, int ninst,
                                  const int *__restrict__ off, const int *__restrict__ cnt,
                                  int *err) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    int inst[3];
    for (int k = 0; k < 3; ++k) {
      const int v = ik[(size_t)k * nelem + e];
      int lo = 0, hi = ninst - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= v) lo = mid; else hi = mid - 1;
      }
      inst[k] = (v >= off[lo] && v < off[lo] + cnt[lo]) ? lo : -1;
    }
    if (inst[0] < 0 || inst[0] != inst[1] || inst[0] != inst[2]) atomicExch(err, 1);
  }
}

}  // namespace bief
