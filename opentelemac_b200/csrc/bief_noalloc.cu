// bief_noalloc.cu -- bief_solve_noalloc: SOLVE (CG, diagonal
// preconditioning) for callers that cannot allocate device memory.
//
// Who needs it: a host code whose device memory is owned by someone else
// -- a Fortran model whose arrays live in OpenACC / OpenMP target data
// regions, a code running under a pool allocator that forbids cudaMalloc
// outside its arena, or a caller that must not trigger the implicit device
// synchronisation cudaMalloc/cudaFree can cause in the middle of its time
// loop.  Such callers already hold IKLE, the matrix and the vectors on the
// device; this entry point solves in place with them and takes every
// other byte it needs from one fixed scratch array compiled into the
// library.
//
// The scratch array is a file-scope static __device__ array of
// NA_SCRATCH_BYTES (about 6.6 MB): every GPU that loads the library holds it
// until the process exits.  It limits the problem to NA_MAX_NPOIN nodes and
// NA_MAX_NELEM elements; larger problems are rejected with BIEF_ERR_SIZE.
// All calls share the array and it keeps the last call's contents, so each
// call clears what must start at zero; calls that overlap on the GPU (two
// streams, two host threads) race on it and must be serialised by the
// caller.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/bief_b200.h"
#include "bief_device.cuh"

using namespace bief;

namespace {

constexpr int NA_MAX_NPOIN = 65536;
constexpr int NA_MAX_NELEM = 131072;
constexpr int NA_THREADS = 1024;
constexpr int NA_MAX_BLOCKS = 1024;

// Scratch layout (byte offsets, each 256-byte aligned).
constexpr size_t al(size_t n) { return (n + 255) & ~size_t(255); }
constexpr size_t OFF_CTL = 0;
constexpr size_t OFF_ERR = OFF_CTL + al(sizeof(Ctl));
constexpr size_t OFF_PTR = OFF_ERR + al(sizeof(int));
constexpr size_t OFF_POS = OFF_PTR + al(sizeof(int) * (NA_MAX_NPOIN + 1));
constexpr size_t OFF_EK = OFF_POS + al(sizeof(int) * NA_MAX_NPOIN);
constexpr size_t OFF_IK = OFF_EK + al(sizeof(int) * 3 * NA_MAX_NELEM);
constexpr size_t OFF_DSC = OFF_IK + al(sizeof(int) * 3 * NA_MAX_NELEM);
constexpr size_t OFF_R = OFF_DSC + al(sizeof(double) * NA_MAX_NPOIN);
constexpr size_t OFF_D0 = OFF_R + al(sizeof(double) * NA_MAX_NPOIN);
constexpr size_t OFF_D1 = OFF_D0 + al(sizeof(double) * NA_MAX_NPOIN);
constexpr size_t OFF_AD = OFF_D1 + al(sizeof(double) * NA_MAX_NPOIN);
constexpr size_t OFF_PART = OFF_AD + al(sizeof(double) * NA_MAX_NPOIN);
constexpr size_t NA_SCRATCH_BYTES = OFF_PART + al(sizeof(double) * 4 * NA_MAX_BLOCKS);

static __device__ __align__(256) unsigned char na_scratch[NA_SCRATCH_BYTES];

// Device address of na_scratch per device, looked up once per device.
std::mutex na_mutex;
void *na_addr[256] = {nullptr};

int na_fail(cudaError_t e, const char *what) {
  fprintf(stderr, "libbief_b200 (noalloc): %s failed (%s)\n", what, cudaGetErrorString(e));
  return BIEF_ERR_CUDA;
}
#define NA_CK(call)                                  \
  do {                                               \
    cudaError_t e__ = (call);                        \
    if (e__ != cudaSuccess) return na_fail(e__, #call); \
  } while (0)

// IKLE(NELMAX,3) 1-based -> 0-based columns (same leading dimension
// NELMAX, so that IKLE and XM share one stride), range check, degrees.
__global__ void k_na_ikle(int npoin, int nelem, int nelmax, const int *__restrict__ ikle, int *ik,
                          int *deg, int *err) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const int v = ikle[(size_t)k * nelmax + e];
      if (v < 1 || v > npoin) {
        atomicExch(err, 1);
        ik[(size_t)k * nelmax + e] = 0;
        continue;
      }
      ik[(size_t)k * nelmax + e] = v - 1;
      atomicAdd(deg + v - 1, 1);
    }
}

// Exclusive scan of the degrees (one block): ptr[0..npoin], pos = ptr.
__global__ void k_na_scan(int npoin, int *deg_pos, int *ptr) {
  __shared__ int part[NA_THREADS];
  const int t = threadIdx.x, T = blockDim.x;
  const int chunk = (npoin + T - 1) / T, lo = min(npoin, t * chunk), hi = min(npoin, lo + chunk);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += deg_pos[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int k = 0; k < T; ++k) {
      const int v = part[k];
      part[k] = run;
      run += v;
    }
    ptr[npoin] = run;
  }
  __syncthreads();
  int run = part[t];
  for (int i = lo; i < hi; ++i) {
    const int d = deg_pos[i];
    ptr[i] = run;
    deg_pos[i] = run;
    run += d;
  }
}

__global__ void k_na_fill(int nelem, int ld, const int *__restrict__ ik, int *pos, int *ek) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const int v = ik[(size_t)k * ld + e];
      ek[atomicAdd(pos + v, 1)] = (e << 2) | k;
    }
}

// Each node's entries in ASSVEC order: local point first, then element
// (assvec.f:88-93); the fill order above is arbitrary, this makes it fixed.
__global__ void k_na_sort(int npoin, const int *__restrict__ ptr, int *ek) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const int j0 = ptr[i], j1 = ptr[i + 1];
    for (int j = j0 + 1; j < j1; ++j) {
      const int v = ek[j];
      const long long key = ((long long)(v & 3) << 32) | (v >> 2);
      int m = j - 1;
      while (m >= j0 && (((long long)(ek[m] & 3) << 32) | (ek[m] >> 2)) > key) {
        ek[m + 1] = ek[m];
        --m;
      }
      ek[m + 1] = v;
    }
  }
}

// PRECD1 (precd1.f:88-158) in place on the caller's arrays, as SOLVE does:
// D = 1/SQRT(DM) guarded, X = X*SQRT(DM), DM = DM*D*D, B = B*D.
__global__ void k_na_precd1_nodes(int npoin, int precon, int td_in, double *dm, double *x,
                                  double *b, double *dsc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npoin; i += gridDim.x * blockDim.x) {
    const double dmi = dm[i];
    double d = precon == 5 ? fabs(dmi) : dmi;
    d = __dsqrt_rn(d);
    x[i] = mul(x[i], d);
    d = (fabs(d) > 1.0e-10) ? __ddiv_rn(1.0, d) : 1.0;
    dsc[i] = d;
    if (td_in == DIA_Q) dm[i] = mul(mul(dmi, d), d);
    else if (td_in == DIA_I) dm[i] = mul(d, d);
    b[i] = mul(b[i], d);
  }
}

// OM1111 'M=DMD' off-diagonals in place (om1111.f:589-603); XM has leading
// dimension nelmax as in the caller's A%X.
__global__ void k_na_precd1_elems(int nelem, int nelmax, int ndiag, const int *__restrict__ ik,
                                  const double *__restrict__ dsc, double *xm) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
    const double d1 = dsc[ik[e]], d2 = dsc[ik[(size_t)nelmax + e]],
                 d3 = dsc[ik[2 * (size_t)nelmax + e]];
    for (int c = 0; c < ndiag; ++c) {
      const int cc = c % 3;
      const double da = cc == 0 ? d2 : d3, db = cc == 2 ? d2 : d1;
      xm[(size_t)c * nelmax + e] = mul(mul(xm[(size_t)c * nelmax + e], da), db);
    }
  }
}

struct NaP {
  int npoin, ld, nitmax;  // ld: leading dimension (NELMAX) of IKLE and XM
  double eps;
  const int *ptr, *ek, *ik;
  const double *xm, *da, *dsc;
  double *x;
  const double *b;
  double *r, *d0, *d1, *ad, *part;
  Ctl *ctl;
  long long timeout_ns;
};

// GRACJG (gracjg.F:169-420), one persistent cooperative launch, rows read
// straight from the EBE arrays (ebe_row) and work vectors in the scratch.
template <int TD, bool SYM>
__global__ void __launch_bounds__(NA_THREADS, 1) k_na_cg(NaP P) {
  const int T = blockDim.x, t = threadIdx.x;
  const int lo = (int)blk_lo(blockIdx.x, P.npoin, gridDim.x);
  const int hi = (int)blk_lo(blockIdx.x + 1, P.npoin, gridDim.x);
  double *x = P.x, *r = P.r, *ad = P.ad;
  const double *b = P.b, *da = P.da;
  const bool lead = (blockIdx.x == 0 && t == 0);
  double s, red;
  int nbar = 0;
  auto row = [&](int i, double acc, auto vec) {
    return ebe_row<double, SYM, false>(i, acc, P.ptr, P.ek, P.ik, P.xm, P.ld, vec);
  };
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
  s = 0.0;
  for (int i = lo + t; i < hi; i += T) s = add(s, mul(b[i], b[i]));
  if (!grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &red, nullptr)) return;
  double xl = red;
  if (__dsqrt_rn(xl) < 1.0e-15) {
    for (int i = lo + t; i < hi; i += T) x[i] = 0.0;
    finish(ST_OK, 0, 0.0, 1.0, 0);
    return;
  }
  int relat = 1;
  if (xl < 1.0) { xl = 1.0; relat = 0; }
  const double tol = mul(xl, mul(P.eps, P.eps));
  s = 0.0;
  for (int i = lo + t; i < hi; i += T) {
    const double ri = sub(row(i, diag_term<TD>(x[i], da, i), [&](int j) { return x[j]; }), b[i]);
    r[i] = ri;
    s = add(s, mul(ri, ri));
  }
  if (!grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &red, nullptr)) return;
  double rmrm = red, rmgm = rmrm;
  if (isnan(rmrm)) { finish(ST_NAN, 0, rmrm, xl, relat); return; }
  if (rmrm < mul(mul(P.eps, P.eps), xl)) { finish(ST_OK, 0, rmrm, xl, relat); return; }
  double *cur = P.d0, *nxt = P.d1;
  s = 0.0;
  for (int i = lo + t; i < hi; i += T) {
    const double di = r[i];
    cur[i] = di;
    const double acc = row(i, diag_term<TD>(di, da, i), [&](int j) { return r[j]; });
    ad[i] = acc;
    s = add(s, mul(di, acc));
  }
  if (!grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &red, nullptr)) return;
  double dad = red;
  if (!(dad > 0.0)) { finish(isnan(dad) ? ST_NAN : ST_BREAKDOWN, 0, rmrm, xl, relat); return; }
  double ro = __ddiv_rn(rmgm, dad);
  for (int m = 1;; ++m) {
    const double nro = -ro;
    s = 0.0;
    for (int i = lo + t; i < hi; i += T) {
      x[i] = add(x[i], mul(nro, cur[i]));
      const double ri = add(r[i], mul(nro, ad[i]));
      r[i] = ri;
      s = add(s, mul(ri, ri));
    }
    if (!grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &red, nullptr)) return;
    const double rm1gm1 = rmgm;
    rmrm = red;
    rmgm = rmrm;
    if (isnan(rmrm)) { finish(ST_NAN, m, rmrm, xl, relat); return; }
    if (rmrm <= tol) { finish(ST_OK, m, rmrm, xl, relat); return; }
    const double beta = __ddiv_rn(rmgm, rm1gm1);
    s = 0.0;
    for (int i = lo + t; i < hi; i += T) {
      const double di = add(r[i], mul(beta, cur[i]));
      nxt[i] = di;
      const double acc = row(i, diag_term<TD>(di, da, i),
                             [&](int j) { return add(r[j], mul(beta, cur[j])); });
      ad[i] = acc;
      s = add(s, mul(di, acc));
    }
    if (!grid_reduce<1, 0>(P.ctl, P.part, P.timeout_ns, nbar, &s, nullptr, &red, nullptr)) return;
    dad = red;
    if (!(dad > 0.0)) { finish(isnan(dad) ? ST_NAN : ST_BREAKDOWN, m, rmrm, xl, relat); return; }
    ro = __ddiv_rn(rmgm, dad);
    double *tmp = cur; cur = nxt; nxt = tmp;
    if (m >= P.nitmax) {
      const double nr = -ro;
      for (int i = lo + t; i < hi; i += T) x[i] = add(x[i], mul(nr, cur[i]));
      finish(m, m, rmrm, xl, relat);
      return;
    }
  }
}

void *na_cg_kernel(int td, bool sym) {
  if (sym) {
    if (td == DIA_Q) return (void *)k_na_cg<DIA_Q, true>;
    if (td == DIA_I) return (void *)k_na_cg<DIA_I, true>;
    return (void *)k_na_cg<DIA_0, true>;
  }
  if (td == DIA_Q) return (void *)k_na_cg<DIA_Q, false>;
  if (td == DIA_I) return (void *)k_na_cg<DIA_I, false>;
  return (void *)k_na_cg<DIA_0, false>;
}

int na_grid(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 16)); }

}  // namespace

extern "C" int bief_solve_noalloc(int npoin, int nelem, int nelmax, const int *ikle, double *dm,
                                  double *xm, char typdia, char typext, double *x, double *b,
                                  bief_slvcfg *cfg, double *relres_out, int device,
                                  void *stream) {
  if (!ikle || !dm || !x || !b || !cfg || npoin <= 0 || nelem <= 0 || nelmax < nelem)
    return BIEF_ERR_ARGS;
  if (npoin > NA_MAX_NPOIN || nelmax > NA_MAX_NELEM) return BIEF_ERR_SIZE;
  const int td_in = (typdia == 'Q' || typdia == 'q') ? DIA_Q
                    : (typdia == 'I' || typdia == 'i') ? DIA_I
                    : typdia == '0' ? DIA_0 : -1;
  if (td_in < 0 || (typext != 'S' && typext != 'Q' && typext != '0')) return BIEF_ERR_ARGS;
  if (typext == '0') return BIEF_ERR_UNSUPPORTED;  // diagonal-only systems: use bief_solve
  if (!xm) return BIEF_ERR_ARGS;
  // the configuration checks of bief_solve, in its order and with its
  // codes, then the one method this entry point runs
  if (cfg->slv < 1 || cfg->slv > 7) return BIEF_ERR_UNSUPPORTED;
  if (cfg->slv == 7 && (cfg->krylov < 1 || cfg->krylov > 20)) return BIEF_ERR_ARGS;
  const int precon = cfg->precon == 0 ? 1 : cfg->precon;
  if (precon <= 0) return BIEF_ERR_ARGS;
  if (precon % 7 == 0 || precon % 11 == 0 || precon % 13 == 0 || precon % 17 == 0)
    return BIEF_ERR_UNSUPPORTED;
  if (cfg->slv != 1) return BIEF_ERR_UNSUPPORTED;
  if (device < 0 || device >= 256) return BIEF_ERR_ARGS;

  int prev = -1;
  NA_CK(cudaGetDevice(&prev));
  if (prev != device) NA_CK(cudaSetDevice(device));
  struct Restore {
    int d;
    ~Restore() {
      if (d >= 0) cudaSetDevice(d);
    }
  } restore{prev != device ? prev : -1};

  unsigned char *base;
  {
    std::lock_guard<std::mutex> lk(na_mutex);
    if (!na_addr[device]) NA_CK(cudaGetSymbolAddress(&na_addr[device], na_scratch));
    base = (unsigned char *)na_addr[device];
  }
  Ctl *ctl = (Ctl *)(base + OFF_CTL);
  int *err = (int *)(base + OFF_ERR);
  int *ptr = (int *)(base + OFF_PTR), *pos = (int *)(base + OFF_POS);
  int *ek = (int *)(base + OFF_EK), *ik = (int *)(base + OFF_IK);
  double *dsc = (double *)(base + OFF_DSC);
  cudaStream_t s = (cudaStream_t)stream;
  int nsm = 0;
  NA_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));

  // gather index of this mesh in the scratch (cleared first: the scratch
  // keeps the previous call's contents)
  NA_CK(cudaMemsetAsync(base, 0, OFF_PTR, s));
  NA_CK(cudaMemsetAsync(pos, 0, sizeof(int) * npoin, s));
  k_na_ikle<<<na_grid(nelem), 256, 0, s>>>(npoin, nelem, nelmax, ikle, ik, pos, err);
  NA_CK(cudaGetLastError());
  int herr = 0;
  NA_CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  NA_CK(cudaStreamSynchronize(s));
  if (herr) return BIEF_ERR_BAD_MESH;
  k_na_scan<<<1, NA_THREADS, 0, s>>>(npoin, pos, ptr);
  k_na_fill<<<na_grid(nelem), 256, 0, s>>>(nelem, nelmax, ik, pos, ek);
  k_na_sort<<<na_grid(npoin), 256, 0, s>>>(npoin, ptr, ek);
  NA_CK(cudaGetLastError());

  // change of variables in place, as SOLVE leaves A and B
  const bool diag = (precon % 2 == 0 || precon % 3 == 0 || precon % 5 == 0);
  int td = td_in;
  if (diag) {
    k_na_precd1_nodes<<<na_grid(npoin), 256, 0, s>>>(npoin, precon, td_in, dm, x, b, dsc);
    const int nd = typext == 'Q' ? 6 : 3;
    k_na_precd1_elems<<<na_grid(nelem), 256, 0, s>>>(nelem, nelmax, nd, ik, dsc, xm);
    td = (td_in == DIA_0) ? DIA_0 : DIA_Q;
    if (precon % 2 == 0 || precon % 3 == 0) td = DIA_I;
    NA_CK(cudaGetLastError());
  }
  void *k = na_cg_kernel(td, typext != 'Q');
  int bps = 0;
  NA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, NA_THREADS, 0));
  if (bps < 1) return BIEF_ERR_CUDA;
  const int need = (npoin + 2 * NA_THREADS - 1) / (2 * NA_THREADS);
  const int G = std::max(1, std::min(std::min(bps * nsm, need), NA_MAX_BLOCKS));
  NaP P;
  P.npoin = npoin;
  P.ld = nelmax;
  P.nitmax = cfg->nitmax;
  P.eps = cfg->eps;
  P.ptr = ptr;
  P.ek = ek;
  P.ik = ik;
  P.xm = xm;
  P.da = dm;
  P.dsc = diag ? dsc : nullptr;
  P.x = x;
  P.b = b;
  P.r = (double *)(base + OFF_R);
  P.d0 = (double *)(base + OFF_D0);
  P.d1 = (double *)(base + OFF_D1);
  P.ad = (double *)(base + OFF_AD);
  P.part = (double *)(base + OFF_PART);
  P.ctl = ctl;
  P.timeout_ns = 2000000000LL;
  void *args[] = {&P};
  NA_CK(cudaLaunchCooperativeKernel(k, dim3(G), dim3(NA_THREADS), args, 0, s));
  Ctl hc;
  NA_CK(cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  NA_CK(cudaStreamSynchronize(s));
  cfg->nit = hc.nit;
  cfg->ok = hc.status == BIEF_OK ? 1 : 0;
  if (relres_out) *relres_out = hc.relres;
  return hc.status;
}
