// bief_device.cuh -- device-side building blocks shared by the BIEF kernels:
// rounding-explicit arithmetic, the fixed dot-product tree, the bounded grid
// barrier of the persistent solvers, and the node-centric EBE row product.
#pragma once

#include <cuda/atomic>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bief {

// ---------------------------------------------------------------------------
// Arithmetic with explicit rounding.  The reference is compiled for x86-64
// without fused multiply-add, so every product and sum is rounded on its own;
// using the _rn intrinsics stops nvcc from contracting a*b+c into an FMA and
// keeps the binary64 path bit-identical to the Fortran.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

// Status codes (same values as include/bief_b200.h).
enum : int {
  ST_OK = 0,
  ST_BREAKDOWN = -2,
  ST_NAN = -3,
  ST_BAD_MESH = -4,
  ST_TIMEOUT = -7,
};

// Diagonal kinds (TYPDIA): 'Q' any, 'I' identity, '0' zero.
enum : int { DIA_Q = 0, DIA_I = 1, DIA_0 = 2 };

// ---------------------------------------------------------------------------
// Fixed-shape block reduction: xor-butterfly inside each warp, warp totals
// (zero-padded to 32) through a second butterfly in warp 0.  The result is
// valid in warp 0.  `sm` holds 32 values.  The CPU oracle restates exactly
// this tree, so dot products are reproducible bit for bit.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T block_tree(T v, T *sm) {
  const unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = add(v, __shfl_xor_sync(FULL, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) sm[w] = v;
  __syncthreads();
  T u = T(0);
  if (w == 0) {
    u = lane < nw ? sm[lane] : T(0);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) u = add(u, __shfl_xor_sync(FULL, u, o));
  }
  __syncthreads();
  return u;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Back-off between polls of a grid barrier's arrival counter (ns).
#ifndef BIEF_SPIN_NS
#define BIEF_SPIN_NS 20
#endif
constexpr unsigned SPIN_NS = BIEF_SPIN_NS;

// Control block of one persistent solve (device memory, zeroed per launch).
struct Ctl {
  unsigned long long arrivals;  // grid-barrier arrivals, never reset in a launch
  int status;                   // final status (written by block 0) or error
  int nit;                      // iterations (CG) / total inner iterations (mixed)
  int relat;                    // 1: relative test, 0: absolute (||B||^2 < 1)
  int outer;                    // mixed: outer refinement steps
  double relres;                // SQRT(RMRM/XL) at exit
};

// Final status of a launch, written by its lead thread.  A block whose
// barrier wait ran out has already stored ST_TIMEOUT (and returned without
// finishing its share of the work); the other blocks may still pass that
// barrier and converge, so the lead only replaces a status that is still
// ST_OK: the host then sees the timeout, never a silently partial result.
__device__ __forceinline__ void set_status(Ctl *ctl, int status) {
  atomicCAS(&ctl->status, (int)ST_OK, status);
}

// Grid-wide reduction + barrier.  Each block reduces its thread partials
// with block_tree (ND binary64 values, NF binary32 values); thread 0 stores
// them in this barrier's half of `part` (two halves used alternately, so a
// block that runs ahead never overwrites partials another block may still
// read) and arrives on a monotonic counter.  The k-th barrier of a launch
// is complete when the counter reaches k*G.  Every block then sums the G
// block partials in block order (thread t: partials t, t+T, ...; then
// block_tree), so all blocks obtain the same bits without a second round
// trip.  The wait is bounded (globaltimer): on timeout the block records
// ST_TIMEOUT and returns false instead of hanging.
// `nbar` counts this block's barriers (uniform across the block).
template <int ND, int NF>
__device__ __noinline__ bool grid_reduce(Ctl *ctl, double *part, long long timeout_ns, int &nbar,
                                         const double *vd, const float *vf, double *od,
                                         float *of) {
  __shared__ double smd[32];
  __shared__ float smf[32];
  __shared__ int s_err;
  constexpr int NV = ND + NF;
  const int G = gridDim.x, T = blockDim.x, t = threadIdx.x;
  const unsigned long long k = (unsigned long long)(++nbar);
  double *buf = part + (size_t)(k & 1) * (size_t)G * NV;
  double bd[ND > 0 ? ND : 1];
  float bf[NF > 0 ? NF : 1];
#pragma unroll
  for (int q = 0; q < ND; ++q) bd[q] = block_tree(vd[q], smd);
#pragma unroll
  for (int q = 0; q < NF; ++q) bf[q] = block_tree(vf[q], smf);
  if (t == 0) {
#pragma unroll
    for (int q = 0; q < ND; ++q) buf[(size_t)blockIdx.x * NV + q] = bd[q];
#pragma unroll
    for (int q = 0; q < NF; ++q) buf[(size_t)blockIdx.x * NV + ND + q] = (double)bf[q];
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
#pragma unroll
  for (int q = 0; q < ND; ++q) {
    double acc = 0.0;
    for (int b = t; b < G; b += T) acc = add(acc, __ldcg(buf + (size_t)b * NV + q));
    od[q] = block_tree(acc, smd);
  }
#pragma unroll
  for (int q = 0; q < NF; ++q) {
    float acc = 0.0f;
    for (int b = t; b < G; b += T) acc = add(acc, (float)__ldcg(buf + (size_t)b * NV + ND + q));
    of[q] = block_tree(acc, smf);
  }
  // block_tree leaves the total in warp 0; broadcast it to the block
  __shared__ double bcd[ND > 0 ? ND : 1];
  __shared__ float bcf[NF > 0 ? NF : 1];
  if (t == 0) {
#pragma unroll
    for (int q = 0; q < ND; ++q) bcd[q] = od[q];
#pragma unroll
    for (int q = 0; q < NF; ++q) bcf[q] = of[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < ND; ++q) od[q] = bcd[q];
#pragma unroll
  for (int q = 0; q < NF; ++q) of[q] = bcf[q];
  __syncthreads();
  return true;
}

// ---------------------------------------------------------------------------
// Compensated dot products (MODASS = 3): Dot2 (dot_comp.f) per thread with
// TWOSUM (twosum.f) and TWOPROD with Dekker's split (twoprod.f, split.f),
// every operation separately rounded; partial results (p, s) merge as
// (p, q) = TwoSum(p1, p2), s = (s1 + s2) + q -- commutative bit for bit, so
// the xor-butterflies leave every lane with the same pair.  Value p + s.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void two_sum(double a, double b, double &x, double &y) {
  const double xo = add(a, b), z = sub(xo, a);
  y = add(sub(a, sub(xo, z)), sub(b, z));
  x = xo;
}

__device__ __forceinline__ void split27(double a, double &hi, double &lo) {
  const double z = mul(134217729.0, a);
  hi = sub(z, sub(z, a));
  lo = sub(a, hi);
}

__device__ __forceinline__ void two_prod(double a, double b, double &x, double &y) {
  double ah, al, bh, bl;
  x = mul(a, b);
  split27(a, ah, al);
  split27(b, bh, bl);
  y = sub(mul(al, bl), sub(sub(sub(x, mul(ah, bh)), mul(al, bh)), mul(ah, bl)));
}

struct CPair {
  double p, s;
};

__device__ __forceinline__ CPair cmerge(CPair a, CPair b) {
  CPair r;
  double q;
  two_sum(a.p, b.p, r.p, q);
  r.s = add(add(a.s, b.s), q);
  return r;
}

// One Dot2 step: (p, s) += x*y
__device__ __forceinline__ void cdot_add(CPair &a, double x, double y) {
  double h, r, q;
  two_prod(x, y, h, r);
  two_sum(a.p, h, a.p, q);
  a.s = add(a.s, add(q, r));
}

__device__ __forceinline__ CPair cpair_shfl_xor(CPair v, int o) {
  const unsigned FULL = 0xffffffffu;
  CPair r;
  r.p = __shfl_xor_sync(FULL, v.p, o);
  r.s = __shfl_xor_sync(FULL, v.s, o);
  return r;
}

__device__ __forceinline__ CPair block_tree_c(CPair v, CPair *sm) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = cmerge(v, cpair_shfl_xor(v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) sm[w] = v;
  __syncthreads();
  CPair u{0.0, 0.0};
  if (w == 0) {
    if (lane < nw) u = sm[lane];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) u = cmerge(u, cpair_shfl_xor(u, o));
  }
  __syncthreads();
  return u;
}

// Grid reduction of one compensated dot, in the order of grid_reduce:
// block pairs (block_tree_c), thread t merging block pairs t, t+T, ...
// from (0, 0), block_tree_c again; returns p + s in `out`.
static __device__ __noinline__ bool grid_reduce_comp(Ctl *ctl, double *part, long long timeout_ns,
                                              int &nbar, CPair v, double *out) {
  __shared__ CPair smc[32];
  __shared__ double bc;
  __shared__ int s_err;
  const int G = gridDim.x, T = blockDim.x, t = threadIdx.x;
  const unsigned long long k = (unsigned long long)(++nbar);
  double *buf = part + (size_t)(k & 1) * (size_t)G * 2;
  const CPair bp = block_tree_c(v, smc);
  if (t == 0) {
    buf[(size_t)blockIdx.x * 2] = bp.p;
    buf[(size_t)blockIdx.x * 2 + 1] = bp.s;
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
  CPair acc{0.0, 0.0};
  for (int b = t; b < G; b += T)
    acc = cmerge(acc, CPair{__ldcg(buf + (size_t)b * 2), __ldcg(buf + (size_t)b * 2 + 1)});
  const CPair tot = block_tree_c(acc, smc);
  if (t == 0) bc = add(tot.p, tot.s);
  __syncthreads();
  *out = bc;
  __syncthreads();
  return true;
}

// Grid reduction of N compensated dots at once (each value exactly as
// grid_reduce_comp reduces it); `part` holds 2 halves of G * 2N doubles.
template <int N>
__device__ __noinline__ bool grid_reduce_comp_n(Ctl *ctl, double *part, long long timeout_ns,
                                                int &nbar, const CPair *v, double *out) {
  __shared__ CPair smc[32];
  __shared__ double bc[N];
  __shared__ int s_err;
  const int G = gridDim.x, T = blockDim.x, t = threadIdx.x;
  const unsigned long long k = (unsigned long long)(++nbar);
  double *buf = part + (size_t)(k & 1) * (size_t)G * 2 * N;
  CPair bp[N];
#pragma unroll
  for (int q = 0; q < N; ++q) bp[q] = block_tree_c(v[q], smc);
  if (t == 0) {
#pragma unroll
    for (int q = 0; q < N; ++q) {
      buf[((size_t)blockIdx.x * N + q) * 2] = bp[q].p;
      buf[((size_t)blockIdx.x * N + q) * 2 + 1] = bp[q].s;
    }
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
#pragma unroll
  for (int q = 0; q < N; ++q) {
    CPair acc{0.0, 0.0};
    for (int b = t; b < G; b += T)
      acc = cmerge(acc, CPair{__ldcg(buf + ((size_t)b * N + q) * 2),
                              __ldcg(buf + ((size_t)b * N + q) * 2 + 1)});
    const CPair tot = block_tree_c(acc, smc);
    if (t == 0) bc[q] = add(tot.p, tot.s);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; ++q) out[q] = bc[q];
  __syncthreads();
  return true;
}

// N dot products accumulated per thread: plain (MODASS = 1: v += x*y, each
// operation rounded) or compensated (MODASS = 3: Dot2 pairs), reduced over
// the grid by dred with the matching tree.
template <bool COMP, int N>
struct DotAcc {
  double v[N];
  CPair c[N];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int q = 0; q < N; ++q) {
      v[q] = 0.0;
      c[q] = CPair{0.0, 0.0};
    }
  }
  __device__ __forceinline__ void acc(int q, double x, double y) {
    if (COMP)
      cdot_add(c[q], x, y);
    else
      v[q] = add(v[q], mul(x, y));
  }
};

template <bool COMP, int N>
__device__ __forceinline__ bool dred(Ctl *ctl, double *part, long long timeout_ns, int &nbar,
                                     const DotAcc<COMP, N> &d, double *out) {
  if constexpr (COMP)
    return grid_reduce_comp_n<N>(ctl, part, timeout_ns, nbar, d.c, out);
  else
    return grid_reduce<N, 0>(ctl, part, timeout_ns, nbar, d.v, nullptr, out, nullptr);
}

// Only the first of an accumulator's N values.
template <bool COMP, int N>
__device__ __forceinline__ bool dred_first(Ctl *ctl, double *part, long long timeout_ns,
                                           int &nbar, const DotAcc<COMP, N> &d, double *out) {
  if constexpr (COMP)
    return grid_reduce_comp_n<1>(ctl, part, timeout_ns, nbar, d.c, out);
  else
    return grid_reduce<1, 0>(ctl, part, timeout_ns, nbar, d.v, nullptr, out, nullptr);
}

// Grid barrier without values: all blocks' preceding writes are visible to
// every block after it returns true.  Same monotonic counter and bounded
// wait as grid_reduce (the two may be mixed in one launch).
static __device__ __noinline__ bool grid_barrier(Ctl *ctl, long long timeout_ns, int &nbar) {
  __shared__ int s_err;
  const unsigned long long k = (unsigned long long)(++nbar);
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> cnt(ctl->arrivals);
    cnt.fetch_add(1ull, cuda::memory_order_release);
    const unsigned long long target = k * (unsigned long long)gridDim.x;
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
  return !s_err;
}

// Plain grid barrier (no values) built on grid_reduce.
__device__ __forceinline__ bool grid_sync(Ctl *ctl, double *part, long long timeout_ns,
                                          int &nbar) {
  double dummy_in = 0.0, dummy_out;
  return grid_reduce<1, 0>(ctl, part, timeout_ns, nbar, &dummy_in, nullptr, &dummy_out, nullptr);
}

// ---------------------------------------------------------------------------
// Node-centric EBE row product.
//
// MV0303 'X=AY' computes per element W1 = XA12*Y(2)+XA13*Y(3),
// W2 = XA23*Y(3)+XA21*Y(1), W3 = XA31*Y(1)+XA32*Y(2) (mv0303.f:123-130) and
// ASSVEC adds W(:,IDP) into X(IKLE(:,IDP)) for IDP=1,2,3 in element order
// (assvec.f:88-93).  For node i that is the left-to-right sum
//   diag_i + sum over (IDP,IELEM) with IKLE(IELEM,IDP)=i of W_IDP(IELEM)
// in (IDP, IELEM) order.  The gather index lists, per node, the packed pairs
// (IELEM<<2 | IDP-1) in exactly that order, so each thread reproduces the
// scatter's additions for its node without atomics.
//
// Column of XM holding XA(k,l) (0-based local points): symmetric storage
// keeps one column per edge (k+l-1); 'Q' storage keeps M12,M13,M23 in
// columns 0..2 and M21,M31,M32 in 3..5 (om1111.f:43-50).
// ---------------------------------------------------------------------------
template <bool SYM>
__device__ __forceinline__ int xm_col(int k, int l) {
  return SYM ? (k + l - 1) : (k < l ? (k + l - 1) : (k + l + 2));
}

// Product W of one gather entry p = (IELEM<<2 | k): the two off-diagonal
// terms of row k of element IELEM times the vector at the element's two
// other points.  DIFF selects the difference form used by the binary32
// inner operator: XA(k,a) (y_a - y_k) + XA(k,b) (y_b - y_k).
template <typename T, bool SYM, bool TRANS, bool DIFF, class V>
__device__ __forceinline__ T entry_product(int p, const int *__restrict__ ik,
                                           const T *__restrict__ xm, int ne, V vec) {
  const int e = p >> 2, k = p & 3;
  const int a = (k == 2) ? 0 : k + 1;  // (k+1) mod 3
  const int b = (k == 0) ? 2 : k - 1;  // (k+2) mod 3
  const int va = __ldg(ik + (size_t)a * ne + e);
  const int vb = __ldg(ik + (size_t)b * ne + e);
  const int ca = TRANS ? xm_col<SYM>(a, k) : xm_col<SYM>(k, a);
  const int cb = TRANS ? xm_col<SYM>(b, k) : xm_col<SYM>(k, b);
  const T xa = __ldg(xm + (size_t)ca * ne + e);
  const T xb = __ldg(xm + (size_t)cb * ne + e);
  if (DIFF) {
    const T yk = vec(__ldg(ik + (size_t)k * ne + e));
    return add(mul(xa, sub(vec(va), yk)), mul(xb, sub(vec(vb), yk)));
  }
  return add(mul(xa, vec(va)), mul(xb, vec(vb)));
}

// EBE row product of node i straight from the element arrays: the node's
// gather entries in ASSVEC order, each W term added left to right.
template <typename T, bool SYM, bool TRANS, class V>
__device__ __forceinline__ T ebe_row(int i, T acc, const int *__restrict__ ptr,
                                     const int *__restrict__ ek, const int *__restrict__ ik,
                                     const T *__restrict__ xm, int ne, V vec) {
  const int j0 = __ldg(ptr + i), j1 = __ldg(ptr + i + 1);
#pragma unroll 2
  for (int j = j0; j < j1; ++j)
    acc = add(acc, entry_product<T, SYM, TRANS, false>(__ldg(ek + j), ik, xm, ne, vec));
  return acc;
}

// ---------------------------------------------------------------------------
// Gather-ready layouts, 32-node slices (sliced ELL): entry m of node i is
// stored at off[i/32] + 32*m + i%32, so the 32 lanes of a warp that own the
// 32 nodes of a slice read consecutive words.
//
// Records (binary64 GRACJG): per gather entry of node i, in ASSVEC order,
// the two coefficients (XA(k,a), XA(k,b)) and the two node numbers (a, b).
// The row product is then exactly the EBE W sum of ebe_row, read as a
// coalesced stream plus two node gathers per entry.
//
// Segments (binary32 inner operator): per distinct neighbour j of node i,
// in order of first appearance among the entries, the binary32 assembled
// coefficient c_ij; product in difference form s_i y_i + sum c_ij (y_j-y_i).
// ---------------------------------------------------------------------------
// Gather entries of one row processed per batch: their index and
// coefficient loads are all issued before the first of their node loads, so
// that a thread keeps SLOT_B dependent load chains in flight (the solvers
// are latency bound: 32 warps per SM at 64 registers).  The additions keep
// their order, so the bits do not depend on the batch sizes.  Measured on
// B200, per iteration at 4.0M / 1.0M nodes: binary64 GRACJG 183 / 51 us with
// 4-entry batches against 207 / 56 us unbatched (6-entry batches: 196 / 54);
// binary32 inner CG 104 / 19.0 us with 6-slot batches against 105 / 19.6
// with 3 and 118 / 21.4 with 5 (interior P1 nodes have 6 neighbours); the
// half-size batch after the full ones takes the binary64 iteration from
// 185 / 51.4 to 183 / 50.8 us and changes nothing on a 1M-point Delaunay
// mesh.
#ifndef BIEF_SLOT_BATCH
#define BIEF_SLOT_BATCH 4
#endif
#ifndef BIEF_SLOT_BATCH32
#define BIEF_SLOT_BATCH32 6
#endif
#ifndef BIEF_SLOT_CASCADE
#define BIEF_SLOT_CASCADE 1
#endif
constexpr int SLOT_B = BIEF_SLOT_BATCH;      // binary64 records
constexpr int SLOT_B32 = BIEF_SLOT_BATCH32;  // binary32 slots
// after the full batches, one batch of half the size when it fits, then
// single entries
constexpr bool SLOT_CASCADE = BIEF_SLOT_CASCADE;

// Loads of the operator streams (binary64 records or segment slots, binary32
// slots): each value is read once per product.  When the kernel's working
// set exceeds the L2 the host sets the stream's flag in Sell and the loads
// are marked evict-first (ld.global.cs), so that the gathered node values,
// reused by every neighbour, keep their place in L2; otherwise they go
// through the read-only path and the whole operator can stay resident.
template <class T>
__device__ __forceinline__ T ld_op(const T *p, int evict_first) {
  return evict_first ? __ldcs(p) : __ldg(p);
}

struct Sell {
  const int *meta;        // per node: gather entries | neighbours << 16
  const int *rec_off;     // per slice: first record
  const int2 *rec_idx;    // per record: (a, b)
  const double2 *rec_c;   // per record: (XA(k,a), XA(k,b)) of the operator
  const int *seg_off;     // per slice: first segment slot
  const int *seg_col;     // per slot: neighbour
  const short *seg_dc;    // per slot: neighbour - node in 16 bits, when every offset fits
  const float *seg_c;     // per slot: binary32 coefficient
  const float *s32;       // per node: binary32 row sum
  const double *sg_c;     // segment storage: per slot, binary64 XA1/XA2
  int cs_rec;             // binary64 operator loads evict-first (ld_op)
  int cs_seg;             // binary32 slot loads evict-first
};

// Two rows at once (nodes i0 and, if has1, i1): independent load chains
// interleaved so that twice as many loads are in flight per thread.  Each
// row's additions keep their own order, so the bits equal rec_row's.
// NB consecutive gather entries m.. of a row: all index/coefficient loads,
// then all node loads, then the additions in order.
template <int NB, class V>
__device__ __forceinline__ void rec_batch(double &a0, const Sell &S, int b0, int m, V vec) {
  double2 c[NB];
  int2 v[NB];
  double ya[NB], yb[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    c[q] = ld_op(S.rec_c + b0 + 32 * (m + q), S.cs_rec);
    v[q] = ld_op(S.rec_idx + b0 + 32 * (m + q), S.cs_rec);
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    ya[q] = vec(v[q].x);
    yb[q] = vec(v[q].y);
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) a0 = add(a0, add(mul(c[q].x, ya[q]), mul(c[q].y, yb[q])));
}

template <class V>
__device__ __forceinline__ void rec_row2(int i0, int i1, bool has1, double &a0, double &a1,
                                         const Sell &S, V vec) {
  if constexpr (SLOT_B > 1) {
    if (!has1) {
      const int d0 = __ldg(S.meta + i0) & 0xffff;
      const int b0 = __ldg(S.rec_off + (i0 >> 5)) + (i0 & 31);
      int m = 0;
      for (; m + SLOT_B <= d0; m += SLOT_B) rec_batch<SLOT_B>(a0, S, b0, m, vec);
      if constexpr (SLOT_CASCADE && SLOT_B / 2 > 1) {
        if (m + SLOT_B / 2 <= d0) {
          rec_batch<SLOT_B / 2>(a0, S, b0, m, vec);
          m += SLOT_B / 2;
        }
      }
      for (; m < d0; ++m) {
        const double2 c = ld_op(S.rec_c + b0 + 32 * m, S.cs_rec);
        const int2 v = ld_op(S.rec_idx + b0 + 32 * m, S.cs_rec);
        a0 = add(a0, add(mul(c.x, vec(v.x)), mul(c.y, vec(v.y))));
      }
      return;
    }
  }
  const int d0 = __ldg(S.meta + i0) & 0xffff;
  const int d1 = has1 ? (__ldg(S.meta + i1) & 0xffff) : 0;
  const int b0 = __ldg(S.rec_off + (i0 >> 5)) + (i0 & 31);
  const int b1 = has1 ? __ldg(S.rec_off + (i1 >> 5)) + (i1 & 31) : 0;
  const int dm = max(d0, d1);
  for (int m = 0; m < dm; ++m) {
    if (m < d0) {
      const double2 c = ld_op(S.rec_c + b0 + 32 * m, S.cs_rec);
      const int2 v = ld_op(S.rec_idx + b0 + 32 * m, S.cs_rec);
      a0 = add(a0, add(mul(c.x, vec(v.x)), mul(c.y, vec(v.y))));
    }
    if (m < d1) {
      const double2 c = ld_op(S.rec_c + b1 + 32 * m, S.cs_rec);
      const int2 v = ld_op(S.rec_idx + b1 + 32 * m, S.cs_rec);
      a1 = add(a1, add(mul(c.x, vec(v.x)), mul(c.y, vec(v.y))));
    }
  }
}

// Segment storage (STO=3, MVSEG order, mvseg.f:129-135): node i has one
// slot per incident segment, in ascending segment order, holding XA1 (node
// is GLOSEG1) or XA2 (GLOSEG2) and the other end, in the sliced layout of
// the binary32 slots (meta, rec_off and seg_col then describe these
// slots).  Row: acc + XA*Y(other) per slot, left to right.
template <int NB, class V>
__device__ __forceinline__ void sgr_batch(double &a0, const Sell &S, int b0, int m, V vec) {
  double c[NB], v[NB];
  int j[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    c[q] = ld_op(S.sg_c + b0 + 32 * (m + q), S.cs_rec);
    j[q] = ld_op(S.seg_col + b0 + 32 * (m + q), S.cs_rec);
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) v[q] = vec(j[q]);
#pragma unroll
  for (int q = 0; q < NB; ++q) a0 = add(a0, mul(c[q], v[q]));
}

template <class V>
__device__ __forceinline__ void sgr_row2(int i0, int i1, bool has1, double &a0, double &a1,
                                         const Sell &S, V vec) {
  if constexpr (SLOT_B > 1) {
    if (!has1) {
      const int d0 = __ldg(S.meta + i0) & 0xffff;
      const int b0 = __ldg(S.rec_off + (i0 >> 5)) + (i0 & 31);
      int m = 0;
      for (; m + SLOT_B <= d0; m += SLOT_B) sgr_batch<SLOT_B>(a0, S, b0, m, vec);
      if constexpr (SLOT_CASCADE && SLOT_B / 2 > 1) {
        if (m + SLOT_B / 2 <= d0) {
          sgr_batch<SLOT_B / 2>(a0, S, b0, m, vec);
          m += SLOT_B / 2;
        }
      }
      for (; m < d0; ++m)
        a0 = add(a0, mul(ld_op(S.sg_c + b0 + 32 * m, S.cs_rec), vec(ld_op(S.seg_col + b0 + 32 * m, S.cs_rec))));
      return;
    }
  }
  const int d0 = __ldg(S.meta + i0) & 0xffff;
  const int d1 = has1 ? (__ldg(S.meta + i1) & 0xffff) : 0;
  const int b0 = __ldg(S.rec_off + (i0 >> 5)) + (i0 & 31);
  const int b1 = has1 ? __ldg(S.rec_off + (i1 >> 5)) + (i1 & 31) : 0;
  const int dm = max(d0, d1);
  for (int m = 0; m < dm; ++m) {
    if (m < d0) a0 = add(a0, mul(ld_op(S.sg_c + b0 + 32 * m, S.cs_rec), vec(ld_op(S.seg_col + b0 + 32 * m, S.cs_rec))));
    if (m < d1) a1 = add(a1, mul(ld_op(S.sg_c + b1 + 32 * m, S.cs_rec), vec(ld_op(S.seg_col + b1 + 32 * m, S.cs_rec))));
  }
}

// Binary64 off-diagonal row product of the working operator in either
// storage: EBE records (STO=1) or segments (STO=3).
template <int STO, class V>
__device__ __forceinline__ void op_row2(int i0, int i1, bool has1, double &a0, double &a1,
                                        const Sell &S, V vec) {
  if constexpr (STO == 3)
    sgr_row2(i0, i1, has1, a0, a1, S, vec);
  else
    rec_row2(i0, i1, has1, a0, a1, S, vec);
}

// Neighbour of binary32 slot r of node i: from the 16-bit offsets (C16, the
// mesh's numbering allowing: 6 instead of 8 bytes per slot) or the column.
template <bool C16>
__device__ __forceinline__ int seg_nb(const Sell &S, int i, int r) {
  if constexpr (C16)
    return i + (int)ld_op(S.seg_dc + r, S.cs_seg);
  else
    return ld_op(S.seg_col + r, S.cs_seg);
}

template <int NB, bool C16, class V>
__device__ __forceinline__ void seg_batch(float &a0, float y0, const Sell &S, int i0, int b0,
                                          int m, V vec) {
  int j[NB];
  float c[NB], v[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    j[q] = seg_nb<C16>(S, i0, b0 + 32 * (m + q));
    c[q] = ld_op(S.seg_c + b0 + 32 * (m + q), S.cs_seg);
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) v[q] = vec(j[q]);
#pragma unroll
  for (int q = 0; q < NB; ++q) a0 = add(a0, mul(c[q], sub(v[q], y0)));
}

// One row of the binary32 product with the node's slot count n0, first
// slot b0 and row sum s already loaded (batched slot loads as below).
template <bool C16, class V>
__device__ __forceinline__ float seg_row_nb(int i0, int n0, int b0, float s, float y0,
                                            const Sell &S, V vec) {
  float a0 = mul(y0, s);
  int m = 0;
  for (; m + SLOT_B32 <= n0; m += SLOT_B32) seg_batch<SLOT_B32, C16>(a0, y0, S, i0, b0, m, vec);
  if constexpr (SLOT_CASCADE && SLOT_B32 / 2 > 1) {
    if (m + SLOT_B32 / 2 <= n0) {
      seg_batch<SLOT_B32 / 2, C16>(a0, y0, S, i0, b0, m, vec);
      m += SLOT_B32 / 2;
    }
  }
  for (; m < n0; ++m) {
    const int jj = seg_nb<C16>(S, i0, b0 + 32 * m);
    const float cc = ld_op(S.seg_c + b0 + 32 * m, S.cs_seg);
    a0 = add(a0, mul(cc, sub(vec(jj), y0)));
  }
  return a0;
}

template <bool C16 = false, class V>
__device__ __forceinline__ void seg_row2(int i0, int i1, bool has1, float y0, float y1,
                                         float &a0, float &a1, const Sell &S, V vec) {
  if constexpr (SLOT_B32 > 1) {
    if (!has1) {
      const int n0 = __ldg(S.meta + i0) >> 16;
      const int b0 = __ldg(S.seg_off + (i0 >> 5)) + (i0 & 31);
      a0 = seg_row_nb<C16>(i0, n0, b0, __ldg(S.s32 + i0), y0, S, vec);
      a1 = 0.0f;
      return;
    }
  }
  const int n0 = __ldg(S.meta + i0) >> 16;
  const int n1 = has1 ? (__ldg(S.meta + i1) >> 16) : 0;
  const int b0 = __ldg(S.seg_off + (i0 >> 5)) + (i0 & 31);
  const int b1 = has1 ? __ldg(S.seg_off + (i1 >> 5)) + (i1 & 31) : 0;
  a0 = mul(y0, __ldg(S.s32 + i0));
  a1 = has1 ? mul(y1, __ldg(S.s32 + i1)) : 0.0f;
  const int nm = max(n0, n1);
  for (int m = 0; m < nm; ++m) {
    if (m < n0) {
      const int j = seg_nb<C16>(S, i0, b0 + 32 * m);
      const float c = ld_op(S.seg_c + b0 + 32 * m, S.cs_seg);
      a0 = add(a0, mul(c, sub(vec(j), y0)));
    }
    if (m < n1) {
      const int j = seg_nb<C16>(S, i1, b1 + 32 * m);
      const float c = ld_op(S.seg_c + b1 + 32 * m, S.cs_seg);
      a1 = add(a1, mul(c, sub(vec(j), y1)));
    }
  }
}

// Single-row forms (the batched solver): the same additions as the
// two-row functions.
template <class V>
__device__ __forceinline__ double rec_row(int i, double acc, const Sell &S, V vec) {
  double unused = 0.0;
  rec_row2(i, i, false, acc, unused, S, vec);
  return acc;
}

template <bool C16 = false, class V>
__device__ __forceinline__ float seg_row(int i, float yi, const Sell &S, V vec) {
  float acc, unused;
  seg_row2<C16>(i, i, false, yi, 0.0f, acc, unused, S, vec);
  return acc;
}

template <int TD, typename T>
__device__ __forceinline__ T diag_term(T yi, const T *__restrict__ da, int i) {
  if (TD == DIA_Q) return mul(yi, da[i]);  // OV 'X=YZ' (mv0303.f:150)
  if (TD == DIA_I) return yi;              // OV 'X=Y'  (mv0303.f:157)
  return T(0);                             // OV 'X=C' with 0 (mv0303.f:159)
}

// Node range of block b of a persistent kernel: [blk_lo(b), blk_lo(b+1)),
// rounded down to multiples of 32 so that warps coincide with slices.
__device__ __forceinline__ long long blk_lo(int b, int n, int nb) {
  return b >= nb ? (long long)n : (((long long)b * n / nb) & ~31LL);
}

}  // namespace bief
