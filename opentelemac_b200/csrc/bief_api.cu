// bief_api.cu -- extern "C" entry points of libbief_b200.so (declared in
// include/bief_b200.h).  Host side of the B200 drop-in for BIEF's
// SOLVE(SLV=1) and MATVEC on EBE P1 matrices: argument validation with the
// reference's semantics, the node->element gather index, device buffers,
// and launches of the kernels in bief_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/bief_b200.h"
#include "bief_batch.cuh"

using namespace bief;

struct bief_handle {
  int dev = 0, npoin = 0, nelem = 0, nelmax = 0, nsm = 0;
  int l2_bytes = 0;  // L2 size of the device (operator-load cache policy)
  cudaStream_t stream = nullptr;
  int G = 0, T = CG_THREADS;  // persistent grid shape (dot tree shape)
  // mesh
  int *d_ptr = nullptr, *d_ek = nullptr, *d_ik = nullptr;
  // stored matrix (A%D, A%X)
  double *d_dm = nullptr, *d_xm = nullptr;
  char typdia = 'Q', typext = 'S';
  int has_matrix = 0;
  // working (scaled) matrix and change of variables
  double *d_dms = nullptr, *d_xms = nullptr, *d_dsc = nullptr;
  // gather-ready layouts (32-node slices): records and binary32 segments
  int *d_meta = nullptr, *d_rec_off = nullptr, *d_seg_off = nullptr, *d_seg_col = nullptr;
  // binary32 slots' neighbours as 16-bit offsets from the node, when every
  // one fits (seg16); the binary32 kernels then read them instead of d_seg_col
  short *d_seg_dc = nullptr;
  bool seg16 = false;
  int2 *d_rec_idx = nullptr;
  uchar2 *d_rec_slot = nullptr;
  // gather records of the standalone MATVEC (Mv16) in format mv16 (MV_*);
  // MV_NONE when a node has more than 255 entries (k_matvec then reads IKLE)
  int mv16 = 0;
  // persistent solvers: twice the resident blocks per SM (bief_set_wide)
  bool wide = false;
  unsigned char *d_mv_deg = nullptr;
  int *d_mv_eb = nullptr;
  void *d_mv_ek = nullptr;  // unsigned short (MV_LOCAL) or int
  void *d_mv_dv = nullptr;  // short2 offsets (MV_LOCAL, MV_BAND); MV_ANY reads d_rec_idx
  double2 *d_rec_c = nullptr;
  double2 *d_rec_ct = nullptr;   // transposed-operator records (EQUNOR, 'Q' storage)
  double *d_sg_ct = nullptr;     // transposed-operator segment slots
  // GMRES: Krylov basis V and A V (2 * krylov * npoin), multi-value partials
  double *d_gmv = nullptr, *d_gpart = nullptr;
  int gm_k = 0;
  float *d_seg_c = nullptr, *d_s32 = nullptr;
  // the stored matrix's generation (bumped on every change) and the one the
  // binary32 copy in d_seg_c / d_sg_c32 / d_s32 was built from (-1: that
  // copy holds a solve's scaled operator)
  long long mat_gen = 0, s32_gen = -1;
  long long nrec = 0, nseg = 0;
  int max_nnb = 0;
  // segment storage (STO=3): GLOSEG, per-node incident segments (sliced),
  // faces of each segment, XA stored and scaled, per-slot coefficients
  int sto = 1, has_segments = 0, nsg = 0;
  long long nsg_slots = 0;
  int *d_g1 = nullptr, *d_g2 = nullptr, *d_sg_meta = nullptr, *d_sg_off = nullptr,
      *d_sg_sx = nullptr, *d_sg_col = nullptr;
  // segment slots' neighbours as 16-bit offsets, when every one fits (sg16)
  short *d_sg_dc = nullptr;
  bool sg16 = false;
  int2 *d_segel = nullptr;
  double *d_xa = nullptr, *d_xas = nullptr, *d_sg_c64 = nullptr;
  float *d_sg_c32 = nullptr;
  // vectors
  double *d_x = nullptr, *d_b = nullptr, *d_bs = nullptr, *d_r = nullptr, *d_d0 = nullptr,
         *d_d1 = nullptr, *d_ad = nullptr, *d_t = nullptr;
  float *d_z = nullptr, *d_ri = nullptr, *d_p0 = nullptr, *d_p1 = nullptr, *d_q = nullptr;
  double *d_part = nullptr, *d_ew = nullptr;
  Ctl *d_ctl = nullptr, *h_ctl = nullptr;
  int *d_err = nullptr;
  // batched solve: per-instance metadata, outputs and tile partials
  int *d_binst = nullptr;      // 3*BATCH_MAX_INST+1 ints (off, n, t0) + outputs
  double *d_brel = nullptr;
  double *d_bpart = nullptr;
  long long bpart_cap = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  float solve_ms = 0.f, matvec_ms = 0.f;
  int mv_pending = 0;
  long long launches = 0;
  long long timeout_ns = 2000000000LL;
};

namespace {

int cuda_fail(cudaError_t e, const char *what, int line) {
  fprintf(stderr, "libbief_b200: %s failed (%s) at %s:%d\n", what, cudaGetErrorString(e), __FILE__,
          line);
  return BIEF_ERR_CUDA;
}
#define CK(call)                                              \
  do {                                                        \
    cudaError_t e__ = (call);                                 \
    if (e__ != cudaSuccess) return cuda_fail(e__, #call, __LINE__); \
  } while (0)

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int typdia_code(char c) {
  switch (c) {
    case 'Q': case 'q': return DIA_Q;
    case 'I': case 'i': return DIA_I;
    case '0': return DIA_0;
    default: return -1;
  }
}

int grid_for(int n, int nsm) {
  int g = (n + 255) / 256;
  return std::max(1, std::min(g, nsm * 16));
}

// One node per thread (MV16_T-thread blocks): the blocks are scheduled as SMs
// free up, so no thread carries a second node into the tail of the launch.
// Used by the EBE MATVECs from compressed records and in binary32 (the
// latter at 4.0M nodes: 47.1 us with 16 resident 256-thread blocks per SM
// looping over the nodes, 43.0 us this way; MVSEG measured no faster).
int mv_grid(int n) { return std::max(1, (n + MV16_T - 1) / MV16_T); }

// Parse an 8-character MATVEC operation string (trailing blanks optional).
int parse_op(const char *op, int *opc, bool *trans) {
  if (!op) return BIEF_ERR_ARGS;
  char s[9];
  int n = 0;
  for (; n < 8 && op[n]; ++n) s[n] = op[n];
  while (n > 0 && s[n - 1] == ' ') --n;
  s[n] = 0;
  struct { const char *name; int opc; bool trans; } tab[] = {
      {"X=AY", OP_AY, false},    {"X=X+AY", OP_XPAY, false}, {"X=-AY", OP_MAY, false},
      {"X=X-AY", OP_XMAY, false}, {"X=X+CAY", OP_XPCAY, false}, {"X=CAY", OP_CAY, false},
      {"X=TAY", OP_AY, true},    {"X=-TAY", OP_MAY, true},   {"X=X+TAY", OP_XPAY, true},
      {"X=X-TAY", OP_XMAY, true}, {"X=X+CTAY", OP_XPCAY, true}};
  for (auto &t : tab)
    if (!strcmp(s, t.name)) {
      *opc = t.opc;
      *trans = t.trans;
      return BIEF_OK;
    }
  return BIEF_ERR_ARGS;
}

template <int TD, bool SYM, bool TR>
void launch_mv(bief_handle *h, const double *xm, const double *da, const double *y, double *x,
               int opc, double c, cudaStream_t st) {
  if (h->mv16) {
    Mv16 M{h->d_mv_deg, h->d_rec_off, h->d_mv_eb, h->d_mv_ek,
           h->mv16 == MV_ANY ? (const void *)h->d_rec_idx : h->d_mv_dv};
    if (h->mv16 == MV_LOCAL)
      k_matvec16<TD, SYM, TR, MV_LOCAL><<<mv_grid(h->npoin), MV16_T, 0, st>>>(
          h->npoin, h->nelem, M, xm, da, y, x, opc, c);
    else if (h->mv16 == MV_BAND)
      k_matvec16<TD, SYM, TR, MV_BAND><<<mv_grid(h->npoin), MV16_T, 0, st>>>(
          h->npoin, h->nelem, M, xm, da, y, x, opc, c);
    else
      k_matvec16<TD, SYM, TR, MV_ANY><<<mv_grid(h->npoin), MV16_T, 0, st>>>(
          h->npoin, h->nelem, M, xm, da, y, x, opc, c);
    return;
  }
  k_matvec<TD, SYM, TR><<<grid_for(h->npoin, h->nsm), 256, 0, st>>>(
      h->npoin, h->nelem, h->d_ptr, h->d_ek, h->d_ik, xm, da, y, x, opc, c);
}

void dispatch_mv(bief_handle *h, int td, bool sym, bool tr, const double *xm, const double *da,
                 const double *y, double *x, int opc, double c, cudaStream_t st) {
#define MV_CASE(TD_, S_, T_) \
  if (td == TD_ && sym == S_ && tr == T_) return launch_mv<TD_, S_, T_>(h, xm, da, y, x, opc, c, st);
  MV_CASE(DIA_Q, true, false) MV_CASE(DIA_I, true, false) MV_CASE(DIA_0, true, false)
  MV_CASE(DIA_Q, false, false) MV_CASE(DIA_I, false, false) MV_CASE(DIA_0, false, false)
  MV_CASE(DIA_Q, true, true) MV_CASE(DIA_I, true, true) MV_CASE(DIA_0, true, true)
  MV_CASE(DIA_Q, false, true) MV_CASE(DIA_I, false, true) MV_CASE(DIA_0, false, true)
#undef MV_CASE
}

// Kernel of a method for TYPDIA code td, storage sto, dot-product mode
// (comp: MODASS = 3, compensated) and residency (wide: twice the blocks per
// SM, MINB = 2 CG_MIN_BLOCKS)
#define KSEL1(k, STO_, C_, M_)                                                \
  (td == DIA_Q ? (void *)k<DIA_Q, STO_, C_, M_>                                \
               : td == DIA_I ? (void *)k<DIA_I, STO_, C_, M_> : (void *)k<DIA_0, STO_, C_, M_>)
#define KSELM(k, M_)                                                          \
  (sto == 3 ? (comp ? KSEL1(k, 3, true, M_) : KSEL1(k, 3, false, M_))         \
            : (comp ? KSEL1(k, 1, true, M_) : KSEL1(k, 1, false, M_)))
#define KSEL(k) (wide ? KSELM(k, 2 * CG_MIN_BLOCKS) : KSELM(k, CG_MIN_BLOCKS))

void *cg_kernel(int td, int sto, bool comp = false, bool wide = false) { return KSEL(k_cg64); }

void *equnor_kernel(int td, int sto, bool comp = false, bool wide = false) {
  return KSEL(k_equnor);
}

void *rescjg_kernel(int td, int sto, bool comp = false, bool wide = false) {
  return KSEL(k_rescjg);
}

void *errmin_kernel(int td, int sto, bool comp = false, bool wide = false) {
  return KSEL(k_errmin);
}

void *cgsqua_kernel(int td, int sto, bool comp = false, bool wide = false) {
  return KSEL(k_cgsqua);
}

void *gmres_kernel(int td, int sto, bool comp = false, bool wide = false) {
  return KSEL(k_gmres);
}

void *cgstab_kernel(int td, int sto, bool comp = false, bool wide = false) {
  return KSEL(k_cgstab);
}

// ... and, for the binary32 kernels, c16: the slots' neighbours as 16-bit
// offsets
#define MSEL1(k, STO_, M_, C_)                                                \
  (td == DIA_Q ? (void *)k<DIA_Q, STO_, M_, C_>                                \
               : td == DIA_I ? (void *)k<DIA_I, STO_, M_, C_> : (void *)k<DIA_0, STO_, M_, C_>)
#define MSELM(k, M_)                                                          \
  (sto == 3 ? (c16 ? MSEL1(k, 3, M_, true) : MSEL1(k, 3, M_, false))          \
            : (c16 ? MSEL1(k, 1, M_, true) : MSEL1(k, 1, M_, false)))
#define MSEL(k) (wide ? MSELM(k, 2 * CG_MIN_BLOCKS) : MSELM(k, CG_MIN_BLOCKS))

void *mixed_kernel(int td, int sto, bool wide = false, bool c16 = false) {
  return MSEL(k_mixed);
}

void *batch_kernel(int td, int sto, bool wide = false, bool c16 = false) {
  return MSEL(k_batch);
}

template <int TD, bool SYM, bool TR>
void launch_mvseg(bief_handle *h, bool ext, const double *xa, const double *da, const double *y,
                  double *x, int opc, double c, cudaStream_t st) {
  k_mvseg<TD, SYM, TR><<<grid_for(h->npoin, h->nsm), 256, 0, st>>>(
      h->npoin, h->nsg, ext, h->d_sg_meta, h->d_sg_off, h->d_sg_sx, h->d_sg_col, xa, da, y, x,
      opc, c);
}

void dispatch_mvseg(bief_handle *h, int td, bool sym, bool tr, bool ext, const double *xa,
                    const double *da, const double *y, double *x, int opc, double c,
                    cudaStream_t st) {
#define MVS_CASE(TD_, S_, T_) \
  if (td == TD_ && sym == S_ && tr == T_) return launch_mvseg<TD_, S_, T_>(h, ext, xa, da, y, x, opc, c, st);
  MVS_CASE(DIA_Q, true, false) MVS_CASE(DIA_I, true, false) MVS_CASE(DIA_0, true, false)
  MVS_CASE(DIA_Q, false, false) MVS_CASE(DIA_I, false, false) MVS_CASE(DIA_0, false, false)
  MVS_CASE(DIA_Q, true, true) MVS_CASE(DIA_I, true, true) MVS_CASE(DIA_0, true, true)
  MVS_CASE(DIA_Q, false, true) MVS_CASE(DIA_I, false, true) MVS_CASE(DIA_0, false, true)
#undef MVS_CASE
}

// Largest grid of the persistent kernels that is guaranteed co-resident,
// reduced for small meshes so that each thread has at least two nodes.
// Automatic residency: two blocks per SM once the binary32 operator and
// vectors (about 80 B per node) exceed 2.25 times the L2.  Measured on the
// B200 (126 MB L2), 400 capped iterations on smooth meshes, one against two
// blocks per SM: binary64 / mixed 33.1 / 14.7 against 36.7 / 16.3 ms at
// 2.0M nodes, 53.9 / 24.9 against 54.0 / 25.3 at 3.0M, 63.6 / 30.4 against
// 62.7 / 30.5 at 3.5M, 71.8 / 37.6 against 71.8 / 35.2 at 4.0M and 93.1 /
// 52.5 against 91.2 / 46.0 at 5.3M.
static bool wide_by_size(int npoin, int l2_bytes) {
  return (double)npoin * 80.0 > 2.25 * (double)l2_bytes;
}

// Cooperative grid of the persistent solvers: the blocks per SM that every
// persistent kernel of this residency can hold at once, times the SMs, but
// no more blocks than rows of two block-widths.
int persistent_grid(int npoin, int nsm, bool wide, int *out) {
  int best = 1 << 30;
  std::vector<void *> ks;
  for (int td : {DIA_Q, DIA_I, DIA_0})
    for (int sto : {1, 3}) {
      ks.push_back(mixed_kernel(td, sto, wide));
      ks.push_back(mixed_kernel(td, sto, wide, true));
      for (bool comp : {false, true})
        for (void *k : {cg_kernel(td, sto, comp, wide), equnor_kernel(td, sto, comp, wide),
                        rescjg_kernel(td, sto, comp, wide), errmin_kernel(td, sto, comp, wide),
                        cgsqua_kernel(td, sto, comp, wide), gmres_kernel(td, sto, comp, wide),
                        cgstab_kernel(td, sto, comp, wide)})
          ks.push_back(k);
    }
  for (void *k : ks) {
    int bps = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, CG_THREADS, 0));
    best = std::min(best, bps);
  }
  if (best < 1) return BIEF_ERR_CUDA;
  int g = best * nsm;
  int need = (npoin + 2 * CG_THREADS - 1) / (2 * CG_THREADS);
  *out = std::max(1, std::min(g, need));
  return BIEF_OK;
}

template <typename T>
int dalloc(T **p, size_t n) {
  CK(cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(n, 1)));
  return BIEF_OK;
}

int ensure_matrix_buffers(bief_handle *h) {
  if (h->d_xm) return BIEF_OK;
  size_t ne = (size_t)h->nelem;
  int st;
  if ((st = dalloc(&h->d_xm, 6 * ne))) return st;
  if ((st = dalloc(&h->d_xms, 6 * ne))) return st;
  return BIEF_OK;
}

void print_gracjg(int status, int nit, double relres, int relat, const char *name = "GRACJG") {
  // gracjg.F:426-435 / equnor.f:317-332 formats (converged, NITMAX)
  if (status > 0)
    printf(" %s (BIEF) : EXCEEDING MAXIMUM ITERATIONS:%8d %s PRECISION:%16.7G\n", name, nit,
           relat ? "RELATIVE" : "ABSOLUTE", relres);
  else
    printf(" %s (BIEF) : %8d ITERATIONS, %s PRECISION:%16.7G\n", name, nit,
           relat ? "RELATIVE" : "ABSOLUTE", relres);
}

int launch_coop(bief_handle *h, void *k, void *arg, cudaStream_t st) {
  void *args[] = {arg};
  CK(cudaLaunchCooperativeKernel(k, dim3(h->G), dim3(h->T), args, 0, st));
  h->launches++;
  return BIEF_OK;
}

// PRECD1 (precd1.f:88-158) into the working matrix; x scaled in place,
// b_out = D*b_in.  Returns the working TYPDIA.
int do_precd1(bief_handle *h, int precon, double *x, const double *b_in, double *b_out,
              int *td_work, cudaStream_t st) {
  const int n = h->npoin;
  const int td_in = typdia_code(h->typdia);
  k_precd1_nodes<<<grid_for(n, h->nsm), 256, 0, st>>>(n, precon, td_in, h->d_dm, x, b_in, b_out,
                                                      h->d_dsc, h->d_dms);
  h->launches++;
  if (h->sto == 3) {
    const int ncol = h->typext == 'Q' ? 2 : (h->typext == 'S' ? 1 : 0);
    if (ncol) {
      k_precd1_segs<<<grid_for(h->nsg, h->nsm), 256, 0, st>>>(h->nsg, ncol, h->d_g1, h->d_g2,
                                                              h->d_dsc, h->d_xa, h->d_xas);
      h->launches++;
    }
  } else {
    const int ndiag = h->typext == 'Q' ? 6 : (h->typext == 'S' ? 3 : 0);
    if (ndiag) {
      k_precd1_elems<<<grid_for(h->nelem, h->nsm), 256, 0, st>>>(h->nelem, ndiag, h->d_ik,
                                                                  h->d_dsc, h->d_xm, h->d_xms);
      h->launches++;
    }
  }
  // TYPDIA after OM 'M=DMD' is 'Q' (unless '0'); PRECON divisible by 2
  // or 3 then makes it the identity (precd1.f:137-142).
  int td = (td_in == DIA_0) ? DIA_0 : DIA_Q;
  if (precon % 2 == 0 || precon % 3 == 0) td = DIA_I;
  *td_work = td;
  CK(cudaGetLastError());
  return BIEF_OK;
}

// Records of the working operator xm (binary64 gather-ready layout).
int build_records(bief_handle *h, const double *xm, cudaStream_t st) {
  const int g = grid_for(h->npoin, h->nsm);
  if (h->typext == 'Q')
    k_build_rec<false><<<g, 256, 0, st>>>(h->npoin, h->nelem, h->d_ptr, h->d_ek, xm, h->d_rec_off,
                                         h->d_rec_c);
  else
    k_build_rec<true><<<g, 256, 0, st>>>(h->npoin, h->nelem, h->d_ptr, h->d_ek, xm, h->d_rec_off,
                                        h->d_rec_c);
  h->launches++;
  CK(cudaGetLastError());
  return BIEF_OK;
}

// Per-slot binary64 coefficients of the working segment operator xa.
int build_seg_coefs(bief_handle *h, const double *xa, cudaStream_t st) {
  const int g = grid_for(h->npoin, h->nsm);
  if (h->typext == 'Q')
    k_build_sgc<false><<<g, 256, 0, st>>>(h->npoin, h->nsg, h->d_sg_meta, h->d_sg_off,
                                         h->d_sg_sx, xa, h->d_sg_c64);
  else
    k_build_sgc<true><<<g, 256, 0, st>>>(h->npoin, h->nsg, h->d_sg_meta, h->d_sg_off,
                                        h->d_sg_sx, xa, h->d_sg_c64);
  h->launches++;
  CK(cudaGetLastError());
  return BIEF_OK;
}

// Transposed-operator coefficients for EQUNOR ('Q' storage; symmetric
// storage reuses the operator's own).  Returns the Sell of A^T.
int build_transposed(bief_handle *h, const double *xm, cudaStream_t st, Sell *out);

// Operator loads are marked evict-first when the kernel's working set --
// the operator stream plus the node vectors the solvers keep (binary64:
// about 7 of 8 B per node; binary32: meta, row sum and 5 vectors of 4 B) --
// exceeds the L2.  Measured on the B200 at 1.0M nodes: binary64 GRACJG
// 97.0 -> 74.0 ms with its 144 MB of records streamed, while the binary32
// mixed solve, whose ~83 MB stay in the 126 MB L2, went from 33.3 to 42.0 ms
// with its slots streamed; at 4.0M nodes streaming both took the mixed solve
// from 682 to 631 ms and binary64 from 1185 to 1164 ms.  Same bits either way.
static void set_cache_policy(const bief_handle *h, Sell &S) {
  const double l2 = (double)h->l2_bytes, n = (double)h->npoin;
  const double op64 = h->sto == 3 ? 12.0 * (double)h->nsg_slots : 24.0 * (double)h->nrec;
  const double op32 = h->sto == 3 ? (h->sg16 ? 6.0 : 8.0) * (double)h->nsg_slots
                                  : (h->seg16 ? 6.0 : 8.0) * (double)h->nseg;
  S.cs_rec = l2 > 0.0 && op64 + 56.0 * n > l2;
  S.cs_seg = l2 > 0.0 && op32 + 28.0 * n > l2;
}

// The binary32 slots of the current storage name their neighbours as
// 16-bit offsets.
static bool slots16(const bief_handle *h) { return h->sto == 3 ? h->sg16 : h->seg16; }

Sell sell_of(const bief_handle *h) {
  Sell S;
  S.sg_c = nullptr;
  set_cache_policy(h, S);
  if (h->sto == 3) {  // segment slots stand in for records and binary32 slots
    S.meta = h->d_sg_meta;
    S.rec_off = h->d_sg_off;
    S.rec_idx = nullptr;
    S.rec_c = nullptr;
    S.seg_off = h->d_sg_off;
    S.seg_col = h->d_sg_col;
    S.seg_dc = h->sg16 ? h->d_sg_dc : nullptr;
    S.seg_c = h->d_sg_c32;
    S.s32 = h->d_s32;
    S.sg_c = h->d_sg_c64;
    return S;
  }
  S.meta = h->d_meta;
  S.rec_off = h->d_rec_off;
  S.rec_idx = h->d_rec_idx;
  S.rec_c = h->d_rec_c;
  S.seg_off = h->d_seg_off;
  S.seg_col = h->d_seg_col;
  S.seg_dc = h->seg16 ? h->d_seg_dc : nullptr;
  S.seg_c = h->d_seg_c;
  S.s32 = h->d_s32;
  return S;
}

int build_transposed(bief_handle *h, const double *xm, cudaStream_t st, Sell *out) {
  Sell S = sell_of(h);
  if (h->typext != 'Q') {
    *out = S;
    return BIEF_OK;
  }
  const int g = grid_for(h->npoin, h->nsm);
  if (h->sto == 3) {
    if (!h->d_sg_ct && dalloc(&h->d_sg_ct, (size_t)h->nsg_slots)) return BIEF_ERR_CUDA;
    k_build_sgc<false, true><<<g, 256, 0, st>>>(h->npoin, h->nsg, h->d_sg_meta, h->d_sg_off,
                                               h->d_sg_sx, xm, h->d_sg_ct);
    S.sg_c = h->d_sg_ct;
  } else {
    if (!h->d_rec_ct && dalloc(&h->d_rec_ct, (size_t)h->nrec)) return BIEF_ERR_CUDA;
    k_build_rec<false, true><<<g, 256, 0, st>>>(h->npoin, h->nelem, h->d_ptr, h->d_ek, xm,
                                               h->d_rec_off, h->d_rec_ct);
    S.rec_c = h->d_rec_ct;
  }
  h->launches++;
  CK(cudaGetLastError());
  *out = S;
  return BIEF_OK;
}

int check_cfg(const bief_slvcfg *cfg, int *precon) {
  if (!cfg) return BIEF_ERR_ARGS;
  if (cfg->slv < 1 || cfg->slv > 7) return BIEF_ERR_UNSUPPORTED;
  if (cfg->slv == 7 && (cfg->krylov < 1 || cfg->krylov > GM_MAXK)) return BIEF_ERR_ARGS;
  int p = cfg->precon == 0 ? 1 : cfg->precon;
  if (p <= 0) return BIEF_ERR_ARGS;
  if (p % 7 == 0 || p % 11 == 0 || p % 13 == 0 || p % 17 == 0) return BIEF_ERR_UNSUPPORTED;
  *precon = p;
  return BIEF_OK;
}

}  // namespace

extern "C" {

const char *bief_strerror(int s) {
  if (s > 0) return "not converged: NITMAX reached";
  switch (s) {
    case BIEF_OK: return "ok";
    case BIEF_ERR_ARGS: return "invalid argument";
    case BIEF_ERR_BREAKDOWN: return "breakdown: D.AD <= 0 (matrix not positive definite)";
    case BIEF_ERR_NAN: return "NaN or Inf in the iteration";
    case BIEF_ERR_BAD_MESH: return "bad mesh: IKLE outside 1..NPOIN or non-positive element area";
    case BIEF_ERR_UNSUPPORTED: return "unsupported solver, preconditioning or storage";
    case BIEF_ERR_CUDA: return "CUDA runtime error";
    case BIEF_ERR_DEVICE_TIMEOUT: return "device barrier wait timed out";
    case BIEF_ERR_NO_MATRIX: return "no matrix set on this handle";
    case BIEF_ERR_SIZE: return "problem size exceeds a fixed limit";
    default: return "unknown status";
  }
}

int bief_mesh_create(int npoin, int nelem, int nelmax, const int *ikle, int device,
                     bief_handle **out) {
  if (!out || !ikle || npoin <= 0 || nelem <= 0 || nelmax < nelem) return BIEF_ERR_ARGS;
  if (nelem > (1 << 29)) return BIEF_ERR_SIZE;
  *out = nullptr;
  // IKLE(NELMAX,3), 1-based -> three 0-based columns; range check.
  std::vector<int> ik(3 * (size_t)nelem);
  std::vector<int> deg(npoin + 1, 0);
  for (int k = 0; k < 3; ++k)
    for (int e = 0; e < nelem; ++e) {
      int v = ikle[(size_t)k * nelmax + e];
      if (v < 1 || v > npoin) return BIEF_ERR_BAD_MESH;
      ik[(size_t)k * nelem + e] = v - 1;
      deg[v]++;
    }
  // Node -> (element, local point) gather index in ASSVEC order: local
  // point outer, element inner (assvec.f:88-93), i.e. sorted by (k, e).
  std::vector<int> ptr(npoin + 1, 0);
  for (int i = 0; i < npoin; ++i) ptr[i + 1] = ptr[i] + deg[i + 1];
  std::vector<int> pos(ptr.begin(), ptr.end() - 1);
  std::vector<int> ek(3 * (size_t)nelem);
  for (int k = 0; k < 3; ++k)
    for (int e = 0; e < nelem; ++e) {
      int v = ik[(size_t)k * nelem + e];
      ek[pos[v]++] = (e << 2) | k;
    }

  // Sliced layouts (32-node slices).  Records: one per gather entry, with
  // its two neighbour nodes.  Segments: the distinct neighbours of each
  // node in order of first appearance among its entries; each record also
  // gets the slots of its two neighbours for the binary32 assembly.
  const int nsl = (npoin + 31) / 32;
  std::vector<int> rec_off(nsl + 1, 0), seg_off(nsl + 1, 0), meta(npoin, 0), nnb(npoin, 0);
  std::vector<int> nb_list;  // per node, consecutive
  std::vector<int> nb_ptr(npoin + 1, 0);
  std::vector<unsigned char> slot_a(3 * (size_t)nelem), slot_b(3 * (size_t)nelem);
  int max_nnb = 0;
  nb_list.reserve(7 * (size_t)npoin);
  for (int i = 0; i < npoin; ++i) {
    const size_t base = nb_list.size();
    for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
      const int e = ek[j] >> 2, k = ek[j] & 3;
      const int va = ik[(size_t)((k + 1) % 3) * nelem + e];
      const int vb = ik[(size_t)((k + 2) % 3) * nelem + e];
      int sl[2];
      const int v2[2] = {va, vb};
      for (int q = 0; q < 2; ++q) {
        size_t t = base;
        while (t < nb_list.size() && nb_list[t] != v2[q]) ++t;
        if (t == nb_list.size()) nb_list.push_back(v2[q]);
        sl[q] = (int)(t - base);
      }
      slot_a[j] = (unsigned char)std::min(sl[0], 255);
      slot_b[j] = (unsigned char)std::min(sl[1], 255);
    }
    nnb[i] = (int)(nb_list.size() - base);
    nb_ptr[i + 1] = (int)nb_list.size();
    max_nnb = std::max(max_nnb, nnb[i]);
    const int d = ptr[i + 1] - ptr[i];
    if (d > 0xffff || nnb[i] > 0x7fff) return BIEF_ERR_SIZE;
    meta[i] = d | (nnb[i] << 16);
  }
  for (int sgi = 0; sgi < nsl; ++sgi) {
    int wr = 0, ws = 0;
    for (int i = 32 * sgi; i < std::min(npoin, 32 * sgi + 32); ++i) {
      wr = std::max(wr, ptr[i + 1] - ptr[i]);
      ws = std::max(ws, nnb[i]);
    }
    const long long r = (long long)rec_off[sgi] + 32LL * wr, q = (long long)seg_off[sgi] + 32LL * ws;
    if (r > 0x7fffffffLL || q > 0x7fffffffLL) return BIEF_ERR_SIZE;
    rec_off[sgi + 1] = (int)r;
    seg_off[sgi + 1] = (int)q;
  }
  const size_t nrec = (size_t)rec_off[nsl], nseg = (size_t)seg_off[nsl];
  std::vector<int2> rec_idx(nrec, make_int2(0, 0));
  std::vector<uchar2> rec_slot(nrec, make_uchar2(0, 0));
  std::vector<int> seg_col(nseg, 0);
  std::vector<short> seg_dc;
  bool seg16 = true;
  for (int i = 0; i < npoin; ++i) {
    const int rb = rec_off[i >> 5] + (i & 31), sb = seg_off[i >> 5] + (i & 31);
    for (int m = 0; m < ptr[i + 1] - ptr[i]; ++m) {
      const int j = ptr[i] + m, e = ek[j] >> 2, k = ek[j] & 3;
      rec_idx[rb + 32 * m] = make_int2(ik[(size_t)((k + 1) % 3) * nelem + e],
                                       ik[(size_t)((k + 2) % 3) * nelem + e]);
      rec_slot[rb + 32 * m] = make_uchar2(slot_a[j], slot_b[j]);
    }
    for (int q = 0; q < nnb[i]; ++q) {
      const int j = nb_list[nb_ptr[i] + q];
      seg_col[sb + 32 * q] = j;
      if (j - i < -32768 || j - i > 32767) seg16 = false;
    }
  }
  if (seg16) {  // the same slots as 16-bit offsets from their node (6 B instead of 8 per slot)
    seg_dc.assign(nseg, 0);
    for (int i = 0; i < npoin; ++i) {
      const int sb = seg_off[i >> 5] + (i & 31);
      for (int q = 0; q < nnb[i]; ++q)
        seg_dc[sb + 32 * q] = (short)(seg_col[sb + 32 * q] - i);
    }
  }

  // MATVEC gather records (Mv16), in the most compact of three formats the
  // mesh allows: MV_LOCAL when, in every slice, the entries' element numbers
  // lie within 2^14 of the slice's smallest and every other vertex within a
  // 16-bit offset of its node (any mesh numbered with some locality: 6 B per
  // entry); MV_BAND when only the vertex offsets fit (8 B); MV_ANY otherwise
  // (12 B: element index and the two vertices, the latter the solver's own
  // rec_idx records).  None when a node has more than 255 entries.
  std::vector<int> mv_eb(nsl, 0);
  bool fit_e = true, fit_v = true, fit_deg = true;
  for (int sgi = 0; sgi < nsl; ++sgi) {
    int lo = INT_MAX, hi = INT_MIN;
    for (int i = 32 * sgi; i < std::min(npoin, 32 * sgi + 32); ++i) {
      if (ptr[i + 1] - ptr[i] > 255) fit_deg = false;
      for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
        lo = std::min(lo, ek[j] >> 2);
        hi = std::max(hi, ek[j] >> 2);
        const int e = ek[j] >> 2, k = ek[j] & 3;
        const long long da = (long long)ik[(size_t)((k + 1) % 3) * nelem + e] - i;
        const long long db = (long long)ik[(size_t)((k + 2) % 3) * nelem + e] - i;
        if (da < -32768 || da > 32767 || db < -32768 || db > 32767) fit_v = false;
      }
    }
    if (lo != INT_MAX && hi - lo >= (1 << 14)) fit_e = false;
    mv_eb[sgi] = lo == INT_MAX ? 0 : lo;
  }
  const int mvf = !fit_deg ? MV_NONE : (fit_e && fit_v) ? MV_LOCAL : fit_v ? MV_BAND : MV_ANY;
  std::vector<unsigned char> mv_deg;
  std::vector<unsigned short> mv_ek16;
  std::vector<int> mv_ek32;
  std::vector<short2> mv_dv16;
  if (mvf != MV_NONE) {
    mv_deg.assign(npoin, 0);
    if (mvf == MV_LOCAL) mv_ek16.assign(nrec, 0); else mv_ek32.assign(nrec, 0);
    if (mvf != MV_ANY) mv_dv16.assign(nrec, make_short2(0, 0));
    for (int i = 0; i < npoin; ++i) {
      const int rb = rec_off[i >> 5] + (i & 31), eb = mv_eb[i >> 5];
      mv_deg[i] = (unsigned char)(ptr[i + 1] - ptr[i]);
      for (int m = 0; m < ptr[i + 1] - ptr[i]; ++m) {
        const int j = ptr[i] + m, e = ek[j] >> 2, k = ek[j] & 3;
        const int va = ik[(size_t)((k + 1) % 3) * nelem + e];
        const int vb = ik[(size_t)((k + 2) % 3) * nelem + e];
        const size_t r = (size_t)rb + 32 * (size_t)m;
        if (mvf == MV_LOCAL) mv_ek16[r] = (unsigned short)(((e - eb) << 2) | k);
        else mv_ek32[r] = ek[j];
        if (mvf != MV_ANY) mv_dv16[r] = make_short2((short)(va - i), (short)(vb - i));
      }
    }
  }

  bief_handle *h = new (std::nothrow) bief_handle;
  if (!h) return BIEF_ERR_ARGS;
  h->dev = device;
  h->npoin = npoin;
  h->nelem = nelem;
  h->nelmax = nelmax;
  h->nrec = (long long)nrec;
  h->nseg = (long long)nseg;
  h->max_nnb = max_nnb;
  int st = BIEF_OK;
  {
    DevGuard g(device);
    auto fail = [&](int s) { bief_destroy(h); return s; };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice", __LINE__));
    if ((e = cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
      return fail(cuda_fail(e, "cudaDeviceGetAttribute", __LINE__));
    if ((e = cudaDeviceGetAttribute(&h->l2_bytes, cudaDevAttrL2CacheSize, device)) != cudaSuccess)
      return fail(cuda_fail(e, "cudaDeviceGetAttribute", __LINE__));
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
      return fail(cuda_fail(e, "cudaStreamCreate", __LINE__));
    for (auto &ev : h->ev)
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail(cuda_fail(e, "cudaEventCreate", __LINE__));
    size_t n = (size_t)npoin, ne = (size_t)nelem;
    if ((st = dalloc(&h->d_ptr, n + 1)) || (st = dalloc(&h->d_ek, 3 * ne)) ||
        (st = dalloc(&h->d_ik, 3 * ne)) || (st = dalloc(&h->d_dm, n)) ||
        (st = dalloc(&h->d_dms, n)) || (st = dalloc(&h->d_dsc, n)) ||
        (st = dalloc(&h->d_s32, n)) || (st = dalloc(&h->d_x, n)) || (st = dalloc(&h->d_b, n)) ||
        (st = dalloc(&h->d_bs, n)) || (st = dalloc(&h->d_r, n)) || (st = dalloc(&h->d_d0, n)) ||
        (st = dalloc(&h->d_d1, n)) || (st = dalloc(&h->d_ad, n)) || (st = dalloc(&h->d_t, n)) ||
        (st = dalloc(&h->d_z, n)) || (st = dalloc(&h->d_ri, n)) || (st = dalloc(&h->d_p0, n)) ||
        (st = dalloc(&h->d_p1, n)) || (st = dalloc(&h->d_q, n)) || (st = dalloc(&h->d_err, 1)) ||
        (st = dalloc(&h->d_ctl, 1)) || (st = dalloc(&h->d_meta, n)) ||
        (st = dalloc(&h->d_rec_off, (size_t)nsl + 1)) || (st = dalloc(&h->d_seg_off, (size_t)nsl + 1)) ||
        (st = dalloc(&h->d_rec_idx, nrec)) || (st = dalloc(&h->d_rec_slot, nrec)) ||
        (st = dalloc(&h->d_rec_c, nrec)) || (st = dalloc(&h->d_seg_col, nseg)) ||
        (st = dalloc(&h->d_seg_c, nseg)))
      return fail(st);
    if (mvf != MV_NONE) {
      const size_t bek = mvf == MV_LOCAL ? sizeof(unsigned short) : sizeof(int);
      const void *hek = mvf == MV_LOCAL ? (const void *)mv_ek16.data() : (const void *)mv_ek32.data();
      unsigned char *dek = nullptr;
      short2 *ddv = nullptr;
      if ((st = dalloc(&h->d_mv_deg, n)) || (st = dalloc(&h->d_mv_eb, (size_t)nsl)))
        return fail(st);
      if ((st = dalloc(&dek, bek * nrec))) return fail(st);
      h->d_mv_ek = dek;
      if (mvf != MV_ANY && (st = dalloc(&ddv, nrec))) return fail(st);
      h->d_mv_dv = ddv;
      if ((e = cudaMemcpyAsync(h->d_mv_deg, mv_deg.data(), n, cudaMemcpyHostToDevice,
                               h->stream)) != cudaSuccess ||
          (e = cudaMemcpyAsync(h->d_mv_eb, mv_eb.data(), sizeof(int) * nsl,
                               cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
          (e = cudaMemcpyAsync(dek, hek, bek * nrec, cudaMemcpyHostToDevice, h->stream)) !=
              cudaSuccess ||
          (mvf != MV_ANY &&
           (e = cudaMemcpyAsync(ddv, mv_dv16.data(), sizeof(short2) * nrec,
                                cudaMemcpyHostToDevice, h->stream)) != cudaSuccess))
        return fail(cuda_fail(e, "mesh upload", __LINE__));
      h->mv16 = mvf;
    }
    if (seg16) {
      if ((st = dalloc(&h->d_seg_dc, (size_t)nseg))) return fail(st);
      if ((e = cudaMemcpyAsync(h->d_seg_dc, seg_dc.data(), sizeof(short) * nseg,
                               cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
        return fail(cuda_fail(e, "mesh upload", __LINE__));
      h->seg16 = true;
    }
    h->wide = wide_by_size(npoin, h->l2_bytes);
    if ((st = persistent_grid(npoin, h->nsm, h->wide, &h->G))) return fail(st);
    if ((st = dalloc(&h->d_part, 8 * (size_t)h->G + 4))) return fail(st);
    if ((e = cudaMallocHost((void **)&h->h_ctl, sizeof(Ctl))) != cudaSuccess)
      return fail(cuda_fail(e, "cudaMallocHost", __LINE__));
    if ((e = cudaMemcpyAsync(h->d_ptr, ptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice,
                             h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_ek, ek.data(), sizeof(int) * 3 * ne, cudaMemcpyHostToDevice,
                             h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_ik, ik.data(), sizeof(int) * 3 * ne, cudaMemcpyHostToDevice,
                             h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_meta, meta.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                             h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_rec_off, rec_off.data(), sizeof(int) * (nsl + 1),
                             cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_seg_off, seg_off.data(), sizeof(int) * (nsl + 1),
                             cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_rec_idx, rec_idx.data(), sizeof(int2) * nrec,
                             cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_rec_slot, rec_slot.data(), sizeof(uchar2) * nrec,
                             cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_seg_col, seg_col.data(), sizeof(int) * nseg,
                             cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_seg_c, 0, sizeof(float) * nseg, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_rec_c, 0, sizeof(double2) * nrec, h->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
      return fail(cuda_fail(e, "mesh upload", __LINE__));
  }
  *out = h;
  return BIEF_OK;
}

int bief_destroy(bief_handle *h) {
  if (!h) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  void *bufs[] = {h->d_ptr, h->d_ek, h->d_ik, h->d_dm, h->d_xm, h->d_dms, h->d_xms, h->d_dsc,
                  h->d_s32, h->d_x, h->d_b, h->d_bs, h->d_r, h->d_d0, h->d_d1,
                  h->d_ad, h->d_t, h->d_z, h->d_ri, h->d_p0, h->d_p1, h->d_q, h->d_part,
                  h->d_ew, h->d_ctl, h->d_err, h->d_meta, h->d_rec_off, h->d_seg_off,
                  h->d_rec_idx, h->d_rec_slot, h->d_rec_c, h->d_seg_col, h->d_seg_dc, h->d_seg_c,
                  h->d_mv_deg, h->d_mv_eb, h->d_mv_ek, h->d_mv_dv,
                  h->d_binst, h->d_brel, h->d_bpart, h->d_g1, h->d_g2, h->d_sg_meta,
                  h->d_sg_off, h->d_sg_sx, h->d_sg_col, h->d_sg_dc, h->d_segel, h->d_xa, h->d_xas,
                  h->d_sg_c64, h->d_sg_c32, h->d_rec_ct, h->d_sg_ct, h->d_gmv, h->d_gpart};
  for (void *p : bufs)
    if (p) cudaFree(p);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  for (auto &ev : h->ev)
    if (ev) cudaEventDestroy(ev);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return BIEF_OK;
}

static int set_matrix_impl(bief_handle *h, const double *dm, const double *xm, char typdia,
                           char typext, bool dev) {
  if (!h || !dm) return BIEF_ERR_ARGS;
  if (typdia_code(typdia) < 0) return BIEF_ERR_ARGS;
  if (typext != 'S' && typext != 'Q' && typext != '0') return BIEF_ERR_ARGS;
  if (typext != '0' && !xm) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  int st = ensure_matrix_buffers(h);
  if (st) return st;
  const size_t n = (size_t)h->npoin, ne = (size_t)h->nelem;
  const int nd = typext == 'Q' ? 6 : (typext == 'S' ? 3 : 0);
  if (dev) {
    CK(cudaMemcpyAsync(h->d_dm, dm, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream));
    if (nd)
      CK(cudaMemcpyAsync(h->d_xm, xm, sizeof(double) * nd * ne, cudaMemcpyDeviceToDevice,
                         h->stream));
  } else {
    CK(cudaMemcpyAsync(h->d_dm, dm, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    if (nd)  // XM(NELMAX,NDIAG) -> leading dimension NELEM
      CK(cudaMemcpy2DAsync(h->d_xm, sizeof(double) * ne, xm, sizeof(double) * h->nelmax,
                           sizeof(double) * ne, nd, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  h->typdia = typdia == 'q' ? 'Q' : (typdia == 'i' ? 'I' : typdia);
  h->typext = typext;
  h->has_matrix = 1;
  h->sto = 1;
  h->mat_gen++;
  return BIEF_OK;
}

int bief_set_matrix(bief_handle *h, const double *dm, const double *xm, char typdia,
                    char typext) {
  return set_matrix_impl(h, dm, xm, typdia, typext, false);
}

int bief_set_matrix_dev(bief_handle *h, const double *dm, const double *xm, char typdia,
                        char typext) {
  return set_matrix_impl(h, dm, xm, typdia, typext, true);
}

int bief_get_matrix(bief_handle *h, double *dm, double *xm, char *typdia) {
  if (!h || !dm) return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  DevGuard g(h->dev);
  const size_t n = (size_t)h->npoin, ne = (size_t)h->nelem;
  CK(cudaMemcpyAsync(dm, h->d_dm, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  if (h->sto == 3) {
    const int nc = h->typext == 'Q' ? 2 : (h->typext == 'S' ? 1 : 0);
    if (nc && xm)
      CK(cudaMemcpyAsync(xm, h->d_xa, sizeof(double) * nc * h->nsg, cudaMemcpyDeviceToHost,
                         h->stream));
  } else {
    const int nd = h->typext == 'Q' ? 6 : (h->typext == 'S' ? 3 : 0);
    if (nd && xm)
      CK(cudaMemcpy2DAsync(xm, sizeof(double) * h->nelmax, h->d_xm, sizeof(double) * ne,
                           sizeof(double) * ne, nd, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  if (typdia) *typdia = h->typdia;
  return BIEF_OK;
}

int bief_get_matrix_dev(bief_handle *h, double *dm, double *xm, void *stream) {
  if (!h || !dm || !xm) return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  DevGuard g(h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)h->npoin, ne = (size_t)h->nelem;
  CK(cudaMemcpyAsync(dm, h->d_dm, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  if (h->sto == 3) {
    const int nc = h->typext == 'Q' ? 2 : (h->typext == 'S' ? 1 : 0);
    if (nc)
      CK(cudaMemcpyAsync(xm, h->d_xa, sizeof(double) * nc * h->nsg, cudaMemcpyDeviceToDevice,
                         st));
  } else {
    const int nd = h->typext == 'Q' ? 6 : (h->typext == 'S' ? 3 : 0);
    if (nd)
      CK(cudaMemcpyAsync(xm, h->d_xm, sizeof(double) * nd * ne, cudaMemcpyDeviceToDevice, st));
  }
  return BIEF_OK;
}

int bief_solve_dev(bief_handle *h, double *x, double *b, bief_slvcfg *cfg, int flags,
                   double *relres_out, void *stream) {
  if (!h || !x || !b) return BIEF_ERR_ARGS;
  int precon, st = check_cfg(cfg, &precon);
  if (st) return st;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  const bool comp = (flags & BIEF_SOLVE_MODASS3) != 0;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  const bool diag = (precon % 2 == 0 || precon % 3 == 0 || precon % 5 == 0);
  int td = typdia_code(h->typdia);
  const bool seg = h->sto == 3;
  const double *xm = seg ? h->d_xa : h->d_xm, *da = h->d_dm;
  const double *bw = b;
  if (diag) {
    if ((st = do_precd1(h, precon, x, b, h->d_bs, &td, s))) return st;
    xm = seg ? h->d_xas : h->d_xms;
    da = h->d_dms;
    bw = h->d_bs;
  }
  if (h->typext == '0') {  // no off-diagonal terms: zero records
    if (seg)
      CK(cudaMemsetAsync(h->d_xas, 0, sizeof(double) * h->nsg, s));
    else
      CK(cudaMemsetAsync(h->d_xms, 0, sizeof(double) * 3 * h->nelem, s));
    xm = seg ? h->d_xas : h->d_xms;
  }
  if ((st = seg ? build_seg_coefs(h, xm, s) : build_records(h, xm, s))) return st;
  CK(cudaMemsetAsync(h->d_ctl, 0, sizeof(Ctl), s));
  // work vectors beyond the handle's own: 2*KRYLOV for GMRES, 3 for CGSTAB,
  // 1 for CGSQUA
  const int nextra =
      cfg->slv == 7 ? 2 * cfg->krylov : (cfg->slv == 6 ? 3 : (cfg->slv == 5 ? 1 : 0));
  if (nextra > 2 * h->gm_k) {
    if (h->d_gmv) cudaFree(h->d_gmv);
    h->d_gmv = nullptr;
    h->gm_k = 0;
    if ((st = dalloc(&h->d_gmv, (size_t)nextra * h->npoin))) return st;
    h->gm_k = (nextra + 1) / 2;
  }
  if (cfg->slv == 6) {  // CGSTAB
    StabP P;
    P.npoin = h->npoin;
    P.nitmax = cfg->nitmax;
    P.eps = cfg->eps;
    P.S = sell_of(h);
    P.da = da;
    P.dsc = diag ? h->d_dsc : nullptr;
    P.x = x;
    P.b = bw;
    P.r = h->d_r;
    P.p = h->d_d0;
    P.q0 = h->d_d1;
    P.q1 = h->d_ad;
    P.v0 = h->d_t;
    P.v1 = h->d_gmv;
    P.s = h->d_gmv + (size_t)h->npoin;
    P.t = h->d_gmv + 2 * (size_t)h->npoin;
    P.part = h->d_part;
    P.ctl = h->d_ctl;
    P.timeout_ns = h->timeout_ns;
    CK(cudaEventRecord(h->ev[0], s));
    if ((st = launch_coop(h, cgstab_kernel(td, h->sto, comp, h->wide), &P, s))) return st;
  } else if (cfg->slv == 7) {  // GMRES
    if (!h->d_gpart && (st = dalloc(&h->d_gpart, 4 * (size_t)h->G * (GM_MAXK + 1) + 4)))
      return st;
    GmP P;
    P.npoin = h->npoin;
    P.nitmax = cfg->nitmax;
    P.krylov = cfg->krylov;
    P.eps = cfg->eps;
    P.S = sell_of(h);
    P.da = da;
    P.dsc = diag ? h->d_dsc : nullptr;
    P.x = x;
    P.b = bw;
    P.r0 = h->d_r;
    P.v = h->d_gmv;
    P.av = h->d_gmv + (size_t)cfg->krylov * h->npoin;
    P.part = h->d_part;
    P.part_n = h->d_gpart;
    P.ctl = h->d_ctl;
    P.timeout_ns = h->timeout_ns;
    CK(cudaEventRecord(h->ev[0], s));
    if ((st = launch_coop(h, gmres_kernel(td, h->sto, comp, h->wide), &P, s))) return st;
  } else if (cfg->slv == 5) {  // CGSQUA
    SquaP P;
    P.npoin = h->npoin;
    P.nitmax = cfg->nitmax;
    P.eps = cfg->eps;
    P.S = sell_of(h);
    P.da = da;
    P.dsc = diag ? h->d_dsc : nullptr;
    P.x = x;
    P.b = bw;
    P.g = h->d_r;
    P.g0 = h->d_gmv;
    P.p = h->d_d0;
    P.k = h->d_d1;
    P.h = h->d_ad;
    P.hk = h->d_t;
    P.part = h->d_part;
    P.ctl = h->d_ctl;
    P.timeout_ns = h->timeout_ns;
    CK(cudaEventRecord(h->ev[0], s));
    if ((st = launch_coop(h, cgsqua_kernel(td, h->sto, comp, h->wide), &P, s))) return st;
  } else if (cfg->slv == 2 || cfg->slv == 4) {  // RESCJG, ERRMIN
    Kry2P P;
    P.npoin = h->npoin;
    P.nitmax = cfg->nitmax;
    P.eps = cfg->eps;
    P.S = sell_of(h);
    P.St = P.S;
    if (cfg->slv == 4 && (st = build_transposed(h, xm, s, &P.St))) return st;
    P.da = da;
    P.dsc = diag ? h->d_dsc : nullptr;
    P.x = x;
    P.b = bw;
    P.r = h->d_r;
    P.d0 = h->d_d0;
    P.d1 = h->d_d1;
    P.ad = h->d_ad;
    P.ag = h->d_t;
    P.part = h->d_part;
    P.ctl = h->d_ctl;
    P.timeout_ns = h->timeout_ns;
    CK(cudaEventRecord(h->ev[0], s));
    void *k = cfg->slv == 2 ? rescjg_kernel(td, h->sto, comp, h->wide) : errmin_kernel(td, h->sto, comp, h->wide);
    if ((st = launch_coop(h, k, &P, s))) return st;
  } else if (cfg->slv == 3) {  // EQUNOR
    EqP P;
    P.npoin = h->npoin;
    P.nitmax = cfg->nitmax;
    P.eps = cfg->eps;
    P.S = sell_of(h);
    if ((st = build_transposed(h, xm, s, &P.St))) return st;
    P.da = da;
    P.dsc = diag ? h->d_dsc : nullptr;
    P.x = x;
    P.b = bw;
    P.r = h->d_r;
    P.d0 = h->d_d0;
    P.d1 = h->d_d1;
    P.ad = h->d_ad;
    P.t = h->d_t;
    P.part = h->d_part;
    P.ctl = h->d_ctl;
    P.timeout_ns = h->timeout_ns;
    CK(cudaEventRecord(h->ev[0], s));
    if ((st = launch_coop(h, equnor_kernel(td, h->sto, comp, h->wide), &P, s))) return st;
  } else {
    CgP P;
    P.npoin = h->npoin;
    P.nitmax = cfg->nitmax;
    P.eps = cfg->eps;
    P.S = sell_of(h);
    P.da = da;
    P.dsc = diag ? h->d_dsc : nullptr;
    P.x = x;
    P.b = bw;
    P.r = h->d_r;
    P.d0 = h->d_d0;
    P.d1 = h->d_d1;
    P.ad = h->d_ad;
    P.part = h->d_part;
    P.ctl = h->d_ctl;
    P.timeout_ns = h->timeout_ns;
    CK(cudaEventRecord(h->ev[0], s));
    if ((st = launch_coop(h, cg_kernel(td, h->sto, comp, h->wide), &P, s))) return st;
  }
  CK(cudaEventRecord(h->ev[1], s));
  CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaEventElapsedTime(&h->solve_ms, h->ev[0], h->ev[1]));
  const Ctl &c = *h->h_ctl;
  st = c.status;
  cfg->nit = c.nit;
  cfg->ok = (st == BIEF_OK) ? 1 : 0;
  if (relres_out) *relres_out = c.relres;
  if (st >= 0 && ((flags & BIEF_SOLVE_INFOGR) || st > 0))
    print_gracjg(st, c.nit, c.relres, c.relat,
                 cfg->slv == 2 ? "RESCJG"
                 : cfg->slv == 3 ? "EQUNOR"
                 : cfg->slv == 4 ? "ERRMIN"
                 : cfg->slv == 5 ? "CGSQUA"
                 : cfg->slv == 6 ? "CGSTAB"
                 : cfg->slv == 7 ? "GMRES" : "GRACJG");
  if (diag && (flags & BIEF_SOLVE_MUTATE_INPUTS) && st >= 0) {
    // SOLVE leaves B = D.B and A = D.A.D with TYPDIA from PRECD1
    h->mat_gen++;
    CK(cudaMemcpyAsync(b, h->d_bs, sizeof(double) * h->npoin, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(h->d_dm, h->d_dms, sizeof(double) * h->npoin, cudaMemcpyDeviceToDevice, s));
    if (seg) {
      const int nc = h->typext == 'Q' ? 2 : (h->typext == 'S' ? 1 : 0);
      if (nc)
        CK(cudaMemcpyAsync(h->d_xa, h->d_xas, sizeof(double) * nc * h->nsg,
                           cudaMemcpyDeviceToDevice, s));
    } else {
      const int nd = h->typext == 'Q' ? 6 : (h->typext == 'S' ? 3 : 0);
      if (nd)
        CK(cudaMemcpyAsync(h->d_xm, h->d_xms, sizeof(double) * nd * h->nelem,
                           cudaMemcpyDeviceToDevice, s));
    }
    CK(cudaStreamSynchronize(s));
    h->typdia = td == DIA_I ? 'I' : (td == DIA_0 ? '0' : 'Q');
  }
  return st;
}

int bief_solve(bief_handle *h, double *x, double *b, bief_slvcfg *cfg, int flags,
               double *relres_out) {
  if (!h || !x || !b) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  const size_t nb = sizeof(double) * h->npoin;
  CK(cudaMemcpyAsync(h->d_x, x, nb, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_b, b, nb, cudaMemcpyHostToDevice, h->stream));
  int st = bief_solve_dev(h, h->d_x, h->d_b, cfg, flags, relres_out, h->stream);
  if (st < 0 && st != BIEF_ERR_BREAKDOWN && st != BIEF_ERR_NAN) return st;
  CK(cudaMemcpyAsync(x, h->d_x, nb, cudaMemcpyDeviceToHost, h->stream));
  if (flags & BIEF_SOLVE_MUTATE_INPUTS)
    CK(cudaMemcpyAsync(b, h->d_b, nb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return st;
}

int bief_solve_mixed_dev(bief_handle *h, double *x, const double *b, int precon,
                         double inner_tol, double outer_tol, int max_outer, int max_inner,
                         int *outer_out, int *inner_out, double *relres_out, void *stream) {
  if (!h || !x || !b || max_inner < 1 || max_outer < 0) return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  if (h->typext != 'S') return BIEF_ERR_UNSUPPORTED;
  if (precon == 0) precon = 1;
  if (precon < 0 || precon % 7 == 0 || precon % 11 == 0 || precon % 13 == 0 || precon % 17 == 0)
    return BIEF_ERR_UNSUPPORTED;
  const bool seg = h->sto == 3;
  if (!seg && h->max_nnb > MAX_NEIGHBOURS) return BIEF_ERR_SIZE;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  const bool diag = (precon % 2 == 0 || precon % 3 == 0 || precon % 5 == 0);
  int td = typdia_code(h->typdia), st;
  const double *xm = seg ? h->d_xa : h->d_xm, *da = h->d_dm, *bw = b;
  if (diag) {
    if ((st = do_precd1(h, precon, x, b, h->d_bs, &td, s))) return st;
    xm = seg ? h->d_xas : h->d_xms;
    da = h->d_dms;
    bw = h->d_bs;
  }
  if (seg) {
    // binary64 slot coefficients, then their binary32 copy and row sums
    if ((st = build_seg_coefs(h, xm, s))) return st;
    const int gn = grid_for(h->npoin, h->nsm);
#define SG_ARGS h->npoin, h->d_sg_meta, h->d_sg_off, h->d_sg_c64, da, h->d_sg_c32, h->d_s32
    if (td == DIA_Q)
      k_build_sg32<DIA_Q><<<gn, 256, 0, s>>>(SG_ARGS);
    else if (td == DIA_I)
      k_build_sg32<DIA_I><<<gn, 256, 0, s>>>(SG_ARGS);
    else
      k_build_sg32<DIA_0><<<gn, 256, 0, s>>>(SG_ARGS);
#undef SG_ARGS
    h->launches++;
    h->s32_gen = -1;
    CK(cudaGetLastError());
  } else if ((st = build_records(h, xm, s))) {
    return st;
  } else {  // binary32 edge-assembled copy of the working operator
    const int gn = grid_for(h->npoin, h->nsm);
#define SEG_ARGS                                                                              \
  h->npoin, h->nelem, h->d_ptr, h->d_ek, xm, da, h->d_meta, h->d_rec_off, h->d_rec_slot, \
      h->d_seg_off, h->d_seg_c, h->d_s32
    if (td == DIA_Q)
      k_build_seg32<DIA_Q><<<gn, 256, 0, s>>>(SEG_ARGS);
    else if (td == DIA_I)
      k_build_seg32<DIA_I><<<gn, 256, 0, s>>>(SEG_ARGS);
    else
      k_build_seg32<DIA_0><<<gn, 256, 0, s>>>(SEG_ARGS);
#undef SEG_ARGS
    h->launches++;
    h->s32_gen = -1;
    CK(cudaGetLastError());
  }
  MixP P;
  P.npoin = h->npoin;
  P.max_outer = max_outer;
  P.max_inner = max_inner;
  P.outer_tol = outer_tol;
  P.inner_tol = inner_tol;
  P.S = sell_of(h);
  P.da = da;
  P.dsc = diag ? h->d_dsc : nullptr;
  P.x = x;
  P.b = bw;
  P.z = h->d_z;
  P.ri = h->d_ri;
  P.p0 = h->d_p0;
  P.p1 = h->d_p1;
  P.q = h->d_q;
  P.part = h->d_part;
  P.ctl = h->d_ctl;
  P.timeout_ns = h->timeout_ns;
  CK(cudaMemsetAsync(h->d_ctl, 0, sizeof(Ctl), s));
  CK(cudaEventRecord(h->ev[0], s));
  if ((st = launch_coop(h, mixed_kernel(td, h->sto, h->wide, slots16(h)), &P, s))) return st;
  CK(cudaEventRecord(h->ev[1], s));
  CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaEventElapsedTime(&h->solve_ms, h->ev[0], h->ev[1]));
  const Ctl &c = *h->h_ctl;
  if (outer_out) *outer_out = c.outer;
  if (inner_out) *inner_out = c.nit;
  if (relres_out) *relres_out = c.relres;
  return c.status;
}

int bief_solve_mixed(bief_handle *h, double *x, const double *b, int precon, double inner_tol,
                     double outer_tol, int max_outer, int max_inner, int *outer_out,
                     int *inner_out, double *relres_out) {
  if (!h || !x || !b) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  const size_t nb = sizeof(double) * h->npoin;
  CK(cudaMemcpyAsync(h->d_x, x, nb, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_b, b, nb, cudaMemcpyHostToDevice, h->stream));
  int st = bief_solve_mixed_dev(h, h->d_x, h->d_b, precon, inner_tol, outer_tol, max_outer,
                                max_inner, outer_out, inner_out, relres_out, h->stream);
  if (st < 0 && st != BIEF_ERR_BREAKDOWN && st != BIEF_ERR_NAN) return st;
  CK(cudaMemcpyAsync(x, h->d_x, nb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return st;
}

int bief_matvec_dev(bief_handle *h, const char *op, double *x, const double *y, double c,
                    void *stream) {
  if (!h || !x || !y) return BIEF_ERR_ARGS;
  int opc;
  bool trans;
  int st = parse_op(op, &opc, &trans);
  if (st) return st;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  const int td = typdia_code(h->typdia);
  const bool sym = h->typext != 'Q';
  const size_t nb = sizeof(double) * h->npoin;
  if (x == y) {  // the reference goes through MESH%T, so X may alias Y
    CK(cudaMemcpyAsync(h->d_t, y, nb, cudaMemcpyDeviceToDevice, s));
    y = h->d_t;
  }
  CK(cudaEventRecord(h->ev[2], s));
  if (h->sto == 3) {  // MVSEG
    dispatch_mvseg(h, td, sym, trans, h->typext != '0', h->d_xa, h->d_dm, y, x, opc, c, s);
  } else {
    const double *xm = h->d_xm;
    if (h->typext == '0') {
      // no off-diagonal terms: reuse the symmetric kernel on a zero operator
      CK(cudaMemsetAsync(h->d_xms, 0, sizeof(double) * 3 * h->nelem, s));
      xm = h->d_xms;
    }
    dispatch_mv(h, td, sym, trans, xm, h->d_dm, y, x, opc, c, s);
  }
  h->launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[3], s));
  h->mv_pending = 1;
  return BIEF_OK;
}

int bief_matvec(bief_handle *h, const char *op, double *x, const double *y, double c) {
  if (!h || !x || !y) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  const size_t nb = sizeof(double) * h->npoin;
  CK(cudaMemcpyAsync(h->d_x, x, nb, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_b, y, nb, cudaMemcpyHostToDevice, h->stream));
  int st = bief_matvec_dev(h, op, h->d_x, h->d_b, c, h->stream);
  if (st) return st;
  CK(cudaMemcpyAsync(x, h->d_x, nb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaEventElapsedTime(&h->matvec_ms, h->ev[2], h->ev[3]));
  h->mv_pending = 0;
  return BIEF_OK;
}

int bief_matvec32_dev(bief_handle *h, float *x, const float *y, void *stream) {
  if (!h || !x || !y) return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  if (h->typext != 'S') return BIEF_ERR_UNSUPPORTED;
  const bool seg = h->sto == 3;
  if (!seg && h->max_nnb > MAX_NEIGHBOURS) return BIEF_ERR_SIZE;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  const int td = typdia_code(h->typdia), gn = grid_for(h->npoin, h->nsm);
  if (h->s32_gen != h->mat_gen) {  // binary32 copy of the stored matrix
    int st;
    if (seg) {
      if ((st = build_seg_coefs(h, h->d_xa, s))) return st;
#define SG_ARGS h->npoin, h->d_sg_meta, h->d_sg_off, h->d_sg_c64, h->d_dm, h->d_sg_c32, h->d_s32
      if (td == DIA_Q)
        k_build_sg32<DIA_Q><<<gn, 256, 0, s>>>(SG_ARGS);
      else if (td == DIA_I)
        k_build_sg32<DIA_I><<<gn, 256, 0, s>>>(SG_ARGS);
      else
        k_build_sg32<DIA_0><<<gn, 256, 0, s>>>(SG_ARGS);
#undef SG_ARGS
    } else {
#define SEG_ARGS                                                                               \
  h->npoin, h->nelem, h->d_ptr, h->d_ek, h->d_xm, h->d_dm, h->d_meta, h->d_rec_off,           \
      h->d_rec_slot, h->d_seg_off, h->d_seg_c, h->d_s32
      if (td == DIA_Q)
        k_build_seg32<DIA_Q><<<gn, 256, 0, s>>>(SEG_ARGS);
      else if (td == DIA_I)
        k_build_seg32<DIA_I><<<gn, 256, 0, s>>>(SEG_ARGS);
      else
        k_build_seg32<DIA_0><<<gn, 256, 0, s>>>(SEG_ARGS);
#undef SEG_ARGS
    }
    h->launches++;
    CK(cudaGetLastError());
    h->s32_gen = h->mat_gen;
  }
  if (x == y) {  // as MATVEC, X may alias Y
    CK(cudaMemcpyAsync(h->d_q, y, sizeof(float) * h->npoin, cudaMemcpyDeviceToDevice, s));
    y = h->d_q;
  }
  CK(cudaEventRecord(h->ev[2], s));
  if (slots16(h))
    k_matvec32<true><<<mv_grid(h->npoin), MV16_T, 0, s>>>(h->npoin, sell_of(h), y, x);
  else
    k_matvec32<false><<<mv_grid(h->npoin), MV16_T, 0, s>>>(h->npoin, sell_of(h), y, x);
  h->launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[3], s));
  h->mv_pending = 1;
  return BIEF_OK;
}

int bief_assemble_wave_dev(bief_handle *h, const double *xc, const double *yc,
                           const double *coef, void *stream) {
  if (!h || !xc || !yc || !coef) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  int st = ensure_matrix_buffers(h);
  if (st) return st;
  if (!h->d_ew && (st = dalloc(&h->d_ew, 4 * (size_t)h->nelem))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(int), s));
  k_wave_elems<<<grid_for(h->nelem, h->nsm), 256, 0, s>>>(h->nelem, h->d_ik, xc, yc, coef,
                                                          h->d_xm, h->d_ew, h->d_err);
  k_wave_nodes<<<grid_for(h->npoin, h->nsm), 256, 0, s>>>(h->npoin, h->d_ptr, h->d_ek, h->nelem,
                                                          h->d_ew, h->d_dm);
  h->launches += 2;
  CK(cudaGetLastError());
  int err = 0;
  CK(cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  h->mat_gen++;
  if (err) return BIEF_ERR_BAD_MESH;
  h->typdia = 'Q';
  h->typext = 'S';
  h->has_matrix = 1;
  h->sto = 1;
  return BIEF_OK;
}

int bief_assemble_mass_diff_dev(bief_handle *h, const double *xc, const double *yc,
                                double xmul_mass, double xmul_dif, int kind, const double *u,
                                const double *v, void *stream) {
  if (!h || !xc || !yc || !u) return BIEF_ERR_ARGS;
  if (kind != 10 && kind != 11 && kind != 12) return BIEF_ERR_ARGS;
  if (kind == 12 && !v) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  int st = ensure_matrix_buffers(h);
  if (st) return st;
  if (!h->d_ew && (st = dalloc(&h->d_ew, 4 * (size_t)h->nelem))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(int), s));
  const int ge = grid_for(h->nelem, h->nsm);
#define MD_ARGS h->nelem, h->d_ik, xc, yc, xmul_mass, xmul_dif, u, v, h->d_xm, h->d_ew, h->d_err
  if (kind == 10)
    k_mass_diff_elems<10><<<ge, 256, 0, s>>>(MD_ARGS);
  else if (kind == 11)
    k_mass_diff_elems<11><<<ge, 256, 0, s>>>(MD_ARGS);
  else
    k_mass_diff_elems<12><<<ge, 256, 0, s>>>(MD_ARGS);
#undef MD_ARGS
  k_wave_nodes<<<grid_for(h->npoin, h->nsm), 256, 0, s>>>(h->npoin, h->d_ptr, h->d_ek, h->nelem,
                                                          h->d_ew, h->d_dm);
  h->launches += 2;
  CK(cudaGetLastError());
  int err = 0;
  CK(cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  h->mat_gen++;
  if (err) return BIEF_ERR_BAD_MESH;
  h->typdia = 'Q';
  h->typext = 'S';
  h->has_matrix = 1;
  h->sto = 1;
  return BIEF_OK;
}

int bief_wave_coef_grad_dev(bief_handle *h, const double *xc, const double *yc,
                            const double *lambda, const double *x, double *grad, void *stream) {
  if (!h || !xc || !yc || !lambda || !x || !grad) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  k_coef_grad<<<grid_for(h->nelem, h->nsm), 256, 0, s>>>(h->nelem, h->d_ik, xc, yc, lambda, x,
                                                         grad);
  h->launches++;
  CK(cudaGetLastError());
  return BIEF_OK;
}

int bief_mass_diff_grad_dev(bief_handle *h, const double *xc, const double *yc,
                            double xmul_dif, int kind, const double *u, const double *v,
                            const double *lambda, const double *x, double *gu, double *gv,
                            void *stream) {
  if (!h || !xc || !yc || !u || !lambda || !x || !gu) return BIEF_ERR_ARGS;
  if (kind != 11 && kind != 12) return BIEF_ERR_ARGS;
  if (kind == 12 && (!v || !gv)) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  int st;
  if (!h->d_ew && (st = dalloc(&h->d_ew, 4 * (size_t)h->nelem))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int ge = grid_for(h->nelem, h->nsm), gn = grid_for(h->npoin, h->nsm);
  if (kind == 11) {
    k_mass_diff_grad_elems<11><<<ge, 256, 0, s>>>(h->nelem, h->d_ik, xc, yc, xmul_dif, u, v,
                                                  lambda, x, h->d_ew);
    k_mass_diff_grad_nodes<11><<<gn, 256, 0, s>>>(h->npoin, h->d_ptr, h->d_ek, h->nelem, h->d_ew,
                                                  u, v, gu, gv);
  } else {
    k_mass_diff_grad_elems<12><<<ge, 256, 0, s>>>(h->nelem, h->d_ik, xc, yc, xmul_dif, u, v,
                                                  lambda, x, h->d_ew);
    k_mass_diff_grad_nodes<12><<<gn, 256, 0, s>>>(h->npoin, h->d_ptr, h->d_ek, h->nelem, h->d_ew,
                                                  u, v, gu, gv);
  }
  h->launches += 2;
  CK(cudaGetLastError());
  return BIEF_OK;
}

int bief_batch_solve_mixed_dev(bief_handle *h, int ninst, const int *node_off,
                               const int *npoin_inst, double *x, const double *b, int precon,
                               double inner_tol, double outer_tol, int max_outer, int max_inner,
                               int nodes_per_thread, int threads_per_block, int *status,
                               int *outer_out,
                               int *inner_out, double *relres_out, void *stream) {
  if (!h || !node_off || !npoin_inst || !x || !b || !status || !outer_out || !inner_out ||
      !relres_out || max_inner < 1 || max_outer < 0)
    return BIEF_ERR_ARGS;
  if (ninst < 1 || ninst > BATCH_MAX_INST) return BIEF_ERR_SIZE;
  if (nodes_per_thread != 1 && nodes_per_thread != 2 && nodes_per_thread != 4 &&
      nodes_per_thread != 8)
    return BIEF_ERR_ARGS;
  if (threads_per_block == 0) threads_per_block = CG_THREADS;
  if (threads_per_block != 256 && threads_per_block != 512 && threads_per_block != 1024)
    return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  if (h->typext != 'S') return BIEF_ERR_UNSUPPORTED;
  const bool seg = h->sto == 3;
  if (!seg && h->max_nnb > MAX_NEIGHBOURS) return BIEF_ERR_SIZE;
  if (precon == 0) precon = 1;
  if (precon < 0 || precon % 7 == 0 || precon % 11 == 0 || precon % 13 == 0 || precon % 17 == 0)
    return BIEF_ERR_UNSUPPORTED;
  // instance ranges: ascending, disjoint, 32-aligned starts, inside the mesh
  const int C = threads_per_block * nodes_per_thread;
  std::vector<int> meta(3 * BATCH_MAX_INST + 1, 0);
  int t0 = 0;
  for (int i = 0; i < ninst; ++i) {
    if (node_off[i] < 0 || node_off[i] % 32 != 0 || npoin_inst[i] < 1 ||
        (long long)node_off[i] + npoin_inst[i] > h->npoin ||
        (i > 0 && node_off[i] < node_off[i - 1] + npoin_inst[i - 1]))
      return BIEF_ERR_ARGS;
    meta[i] = node_off[i];
    meta[BATCH_MAX_INST + i] = npoin_inst[i];
    meta[2 * BATCH_MAX_INST + i] = t0;
    t0 += (npoin_inst[i] + C - 1) / C;
  }
  meta[2 * BATCH_MAX_INST + ninst] = t0;
  const int ntiles = t0;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  int st;
  if (!h->d_binst && ((st = dalloc(&h->d_binst, 7 * (size_t)BATCH_MAX_INST + 1)) ||
                      (st = dalloc(&h->d_brel, (size_t)BATCH_MAX_INST))))
    return st;
  if (h->bpart_cap < 4LL * ntiles) {
    if (h->d_bpart) CK(cudaFree(h->d_bpart));
    h->d_bpart = nullptr;
    if ((st = dalloc(&h->d_bpart, 4 * (size_t)ntiles))) return st;
    h->bpart_cap = 4LL * ntiles;
  }
  int *d_off = h->d_binst, *d_cnt = h->d_binst + BATCH_MAX_INST,
      *d_t0 = h->d_binst + 2 * BATCH_MAX_INST, *d_st = h->d_binst + 3 * BATCH_MAX_INST + 1,
      *d_in = d_st + BATCH_MAX_INST, *d_out = d_in + BATCH_MAX_INST;
  CK(cudaMemcpyAsync(h->d_binst, meta.data(), sizeof(int) * (3 * BATCH_MAX_INST + 1),
                     cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(int), s));
  k_check_blockdiag<<<grid_for(h->nelem, h->nsm), 256, 0, s>>>(h->nelem, h->d_ik, ninst, d_off,
                                                               d_cnt, h->d_err);
  h->launches++;
  int err = 0;
  CK(cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (err) return BIEF_ERR_ARGS;

  const bool diag = (precon % 2 == 0 || precon % 3 == 0 || precon % 5 == 0);
  int td = typdia_code(h->typdia);
  const double *xm = seg ? h->d_xa : h->d_xm, *da = h->d_dm, *bw = b;
  if (diag) {
    if ((st = do_precd1(h, precon, x, b, h->d_bs, &td, s))) return st;
    xm = seg ? h->d_xas : h->d_xms;
    da = h->d_dms;
    bw = h->d_bs;
  }
  if (seg) {
    // segment storage: binary64 slot coefficients, their binary32 copy and
    // row sums, as the single-mesh mixed solve builds them
    if ((st = build_seg_coefs(h, xm, s))) return st;
    const int gn = grid_for(h->npoin, h->nsm);
#define SG_ARGS h->npoin, h->d_sg_meta, h->d_sg_off, h->d_sg_c64, da, h->d_sg_c32, h->d_s32
    if (td == DIA_Q)
      k_build_sg32<DIA_Q><<<gn, 256, 0, s>>>(SG_ARGS);
    else if (td == DIA_I)
      k_build_sg32<DIA_I><<<gn, 256, 0, s>>>(SG_ARGS);
    else
      k_build_sg32<DIA_0><<<gn, 256, 0, s>>>(SG_ARGS);
#undef SG_ARGS
    h->launches++;
    h->s32_gen = -1;
    CK(cudaGetLastError());
  } else if ((st = build_records(h, xm, s))) {
    return st;
  } else {
    const int gn = grid_for(h->npoin, h->nsm);
#define SEG_ARGS                                                                              \
  h->npoin, h->nelem, h->d_ptr, h->d_ek, xm, da, h->d_meta, h->d_rec_off, h->d_rec_slot, \
      h->d_seg_off, h->d_seg_c, h->d_s32
    if (td == DIA_Q)
      k_build_seg32<DIA_Q><<<gn, 256, 0, s>>>(SEG_ARGS);
    else if (td == DIA_I)
      k_build_seg32<DIA_I><<<gn, 256, 0, s>>>(SEG_ARGS);
    else
      k_build_seg32<DIA_0><<<gn, 256, 0, s>>>(SEG_ARGS);
#undef SEG_ARGS
    h->launches++;
    h->s32_gen = -1;
    CK(cudaGetLastError());
  }
  void *k = batch_kernel(td, seg ? 3 : 1, h->wide, seg ? h->sg16 : h->seg16);
  int bps = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, threads_per_block, 0));
  if (bps < 1) return BIEF_ERR_CUDA;
  const int G = std::max(1, std::min(bps * h->nsm, ntiles));
  BatchP P;
  P.ninst = ninst;
  P.npt = nodes_per_thread;
  P.max_outer = max_outer;
  P.max_inner = max_inner;
  P.outer_tol = outer_tol;
  P.inner_tol = inner_tol;
  P.inst_off = d_off;
  P.inst_n = d_cnt;
  P.inst_t0 = d_t0;
  P.S = sell_of(h);
  P.da = da;
  P.dsc = diag ? h->d_dsc : nullptr;
  P.x = x;
  P.b = bw;
  P.z = h->d_z;
  P.ri = h->d_ri;
  P.p0 = h->d_p0;
  P.p1 = h->d_p1;
  P.q = h->d_q;
  P.part = h->d_bpart;
  P.ntiles = ntiles;
  P.ctl = h->d_ctl;
  P.st_out = d_st;
  P.inner_out = d_in;
  P.outer_out = d_out;
  P.relres_out = h->d_brel;
  P.timeout_ns = h->timeout_ns;
  CK(cudaMemsetAsync(h->d_ctl, 0, sizeof(Ctl), s));
  CK(cudaEventRecord(h->ev[0], s));
  void *args[] = {&P};
  CK(cudaLaunchCooperativeKernel(k, dim3(G), dim3(threads_per_block), args, 0, s));
  h->launches++;
  CK(cudaEventRecord(h->ev[1], s));
  CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(status, d_st, sizeof(int) * ninst, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(inner_out, d_in, sizeof(int) * ninst, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(outer_out, d_out, sizeof(int) * ninst, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(relres_out, h->d_brel, sizeof(double) * ninst, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaEventElapsedTime(&h->solve_ms, h->ev[0], h->ev[1]));
  if (h->h_ctl->status == ST_TIMEOUT) return BIEF_ERR_DEVICE_TIMEOUT;
  return BIEF_OK;
}

int bief_diri01_dev(bief_handle *h, int nptfr, const int *nbor, const int *limdir, int kdir,
                    const double *fbor, double *sm, double *f, const double *maskpt,
                    void *stream) {
  if (!h || nptfr < 0 || (nptfr > 0 && (!nbor || !limdir || !fbor)) || !sm || !f)
    return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  const int n = h->npoin, gn = grid_for(n, h->nsm), gb = grid_for(std::max(nptfr, 1), h->nsm);
  double *w1 = h->d_t, *w2 = h->d_ad;
  const int td = typdia_code(h->typdia);
  const bool sym = h->typext != 'Q';
  CK(cudaMemsetAsync(w1, 0, sizeof(double) * n, s));
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(int), s));
  if (nptfr > 0) k_diri_scatter<<<gb, 256, 0, s>>>(nptfr, n, nbor, limdir, kdir, fbor, w1, h->d_err);
  // W2 = S W1 (MATVEC 'X=AY')
  if (h->sto == 3) {
    dispatch_mvseg(h, td, sym, false, h->typext != '0', h->d_xa, h->d_dm, w1, w2, OP_AY, 0.0, s);
  } else {
    const double *xm = h->d_xm;
    if (h->typext == '0') {
      CK(cudaMemsetAsync(h->d_xms, 0, sizeof(double) * 3 * h->nelem, s));
      xm = h->d_xms;
    }
    dispatch_mv(h, td, sym, false, xm, h->d_dm, w1, w2, OP_AY, 0.0, s);
  }
  k_diri_nodes<<<gn, 256, 0, s>>>(n, sm, w2);
  if (nptfr > 0)
    k_diri_aux<<<gb, 256, 0, s>>>(nptfr, n, nbor, limdir, kdir, fbor, h->d_dm, sm, w2, f);
  if (maskpt) k_diri_mask<<<gn, 256, 0, s>>>(n, maskpt, sm, f, w2);
  // OM 'M=DMD' with D = W2 on the off-diagonal terms only, in place
  if (h->sto == 3) {
    const int ncol = h->typext == 'Q' ? 2 : (h->typext == 'S' ? 1 : 0);
    if (ncol)
      k_precd1_segs<<<grid_for(h->nsg, h->nsm), 256, 0, s>>>(h->nsg, ncol, h->d_g1, h->d_g2, w2,
                                                             h->d_xa, h->d_xa);
  } else {
    const int ndiag = h->typext == 'Q' ? 6 : (h->typext == 'S' ? 3 : 0);
    if (ndiag)
      k_precd1_elems<<<grid_for(h->nelem, h->nsm), 256, 0, s>>>(h->nelem, ndiag, h->d_ik, w2,
                                                                h->d_xm, h->d_xm);
  }
  h->launches += 6;
  h->mat_gen++;
  CK(cudaGetLastError());
  if (nptfr > 0) {  // an NBOR entry outside 1..NPOIN was skipped
    int err = 0;
    CK(cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (err) return BIEF_ERR_BAD_MESH;
  }
  return BIEF_OK;
}

int bief_diri01(bief_handle *h, int nptfr, const int *nbor, const int *limdir, int kdir,
                const double *fbor, double *sm, double *f, const double *maskpt) {
  if (!h || nptfr < 0 || !sm || !f) return BIEF_ERR_ARGS;
  if (nptfr > 0 && (!nbor || !limdir || !fbor)) return BIEF_ERR_ARGS;
  for (int k = 0; k < nptfr; ++k)
    if (nbor[k] < 1 || nbor[k] > h->npoin) return BIEF_ERR_BAD_MESH;
  DevGuard g(h->dev);
  const size_t nb = sizeof(double) * h->npoin;
  int *d_i = nullptr;
  double *d_f = nullptr, *d_m = nullptr;
  int st = BIEF_OK;
  if ((st = dalloc(&d_i, 2 * (size_t)nptfr)) || (st = dalloc(&d_f, (size_t)nptfr)) ||
      (maskpt && (st = dalloc(&d_m, (size_t)h->npoin)))) {
    cudaFree(d_i);
    cudaFree(d_f);
    return st;
  }
  cudaError_t e = cudaSuccess;
  if (nptfr > 0) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_i, nbor, sizeof(int) * nptfr, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_i + nptfr, limdir, sizeof(int) * nptfr, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, fbor, sizeof(double) * nptfr, cudaMemcpyHostToDevice, h->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_x, sm, nb, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_b, f, nb, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && maskpt) e = cudaMemcpyAsync(d_m, maskpt, nb, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    st = bief_diri01_dev(h, nptfr, d_i, d_i + nptfr, kdir, d_f, h->d_x, h->d_b, d_m, h->stream);
    if (st == BIEF_OK) {
      e = cudaMemcpyAsync(sm, h->d_x, nb, cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(f, h->d_b, nb, cudaMemcpyDeviceToHost, h->stream);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_i);
  cudaFree(d_f);
  if (d_m) cudaFree(d_m);
  if (e != cudaSuccess) return cuda_fail(e, "bief_diri01", __LINE__);
  return st;
}

int bief_selftest_timeout(int device, long long timeout_ns) {
  if (timeout_ns < 1000000LL || timeout_ns > 5000000000LL) return BIEF_ERR_ARGS;
  DevGuard g(device);
  Ctl *ctl = nullptr;
  CK(cudaMalloc((void **)&ctl, sizeof(Ctl)));
  Ctl host;
  cudaError_t e = cudaMemset(ctl, 0, sizeof(Ctl));
  if (e == cudaSuccess) {
    k_selftest_wait<<<1, 32>>>(ctl, timeout_ns);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&host, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
  cudaFree(ctl);
  if (e != cudaSuccess) return cuda_fail(e, "selftest", __LINE__);
  return host.status == ST_TIMEOUT ? BIEF_ERR_DEVICE_TIMEOUT : BIEF_ERR_CUDA;
}

int bief_launch_info(bief_handle *h, int *nblocks, int *nthreads) {
  if (!h) return BIEF_ERR_ARGS;
  if (nblocks) *nblocks = h->G;
  if (nthreads) *nthreads = h->T;
  return BIEF_OK;
}

int bief_set_blocks_per_sm(bief_handle *h, int blocks_per_sm) {
  if (!h || blocks_per_sm < 0 || blocks_per_sm > 2) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  const bool wide = blocks_per_sm == 0 ? wide_by_size(h->npoin, h->l2_bytes)
                                       : blocks_per_sm == 2;
  int G = 0, st;
  if ((st = persistent_grid(h->npoin, h->nsm, wide, &G))) return st;
  if (G != h->G) {
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaFree(h->d_part));
    h->d_part = nullptr;
    if (h->d_gpart) CK(cudaFree(h->d_gpart));  // sized by G at its first use
    h->d_gpart = nullptr;
    if ((st = dalloc(&h->d_part, 8 * (size_t)G + 4))) return st;
    h->G = G;
  }
  h->wide = wide;
  return BIEF_OK;
}

int bief_matvec_format(bief_handle *h, int *format) {
  if (!h || !format) return BIEF_ERR_ARGS;
  *format = h->mv16;
  return BIEF_OK;
}

int bief_set_segments(bief_handle *h, int nseg, int maxseg, const int *gloseg) {
  if (!h || !gloseg || nseg <= 0 || maxseg < nseg) return BIEF_ERR_ARGS;
  const int n = h->npoin, ne = h->nelem;
  std::vector<int> g1(nseg), g2(nseg);
  for (int s = 0; s < nseg; ++s) {
    const int a = gloseg[s], b = gloseg[(size_t)maxseg + s];
    if (a < 1 || a > n || b < 1 || b > n || a == b) return BIEF_ERR_BAD_MESH;
    g1[s] = a - 1;
    g2[s] = b - 1;
  }
  // Element faces -> segments (face f joins local points f and f+1 mod 3);
  // per segment its faces in element order (at most two).
  std::vector<long long> key(nseg);
  std::vector<int> ord(nseg);
  for (int s = 0; s < nseg; ++s) {
    key[s] = (long long)std::min(g1[s], g2[s]) * n + std::max(g1[s], g2[s]);
    ord[s] = s;
  }
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return key[a] < key[b]; });
  for (int q = 1; q < nseg; ++q)
    if (key[ord[q]] == key[ord[q - 1]]) return BIEF_ERR_BAD_MESH;  // duplicated edge
  std::vector<long long> skey(nseg);
  for (int q = 0; q < nseg; ++q) skey[q] = key[ord[q]];
  std::vector<int2> segel(nseg, make_int2(-1, -1));
  std::vector<int> ik(3 * (size_t)ne);
  if (cudaMemcpy(ik.data(), h->d_ik, sizeof(int) * 3 * (size_t)ne, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return BIEF_ERR_CUDA;
  for (int e = 0; e < ne; ++e)
    for (int f = 0; f < 3; ++f) {
      const int a = ik[(size_t)f * ne + e], b = ik[(size_t)((f + 1) % 3) * ne + e];
      const long long k = (long long)std::min(a, b) * n + std::max(a, b);
      auto it = std::lower_bound(skey.begin(), skey.end(), k);
      if (it == skey.end() || *it != k) return BIEF_ERR_BAD_MESH;  // face without segment
      const int s = ord[it - skey.begin()];
      if (segel[s].x < 0)
        segel[s].x = (e << 2) | f;
      else if (segel[s].y < 0)
        segel[s].y = (e << 2) | f;
      else
        return BIEF_ERR_BAD_MESH;  // edge of more than two elements
    }
  // Per node, incident segments in ascending order (the order in which MVSEG
  // adds into the node), in 32-node slices.
  std::vector<int> deg(n, 0);
  for (int s = 0; s < nseg; ++s) {
    deg[g1[s]]++;
    deg[g2[s]]++;
  }
  const int nsl = (n + 31) / 32;
  std::vector<int> off(nsl + 1, 0), meta(n);
  for (int sl = 0; sl < nsl; ++sl) {
    int w = 0;
    for (int i = 32 * sl; i < std::min(n, 32 * sl + 32); ++i) w = std::max(w, deg[i]);
    const long long o = (long long)off[sl] + 32LL * w;
    if (o > 0x7fffffffLL) return BIEF_ERR_SIZE;
    off[sl + 1] = (int)o;
  }
  for (int i = 0; i < n; ++i) {
    if (deg[i] > 0x7fff) return BIEF_ERR_SIZE;
    meta[i] = deg[i] | (deg[i] << 16);
  }
  const size_t nslot = (size_t)off[nsl];
  std::vector<int> sx(nslot, 0), col(nslot, 0), fill(n, 0);
  std::vector<short> dc(nslot, 0);
  bool fit16 = true;
  for (int s = 0; s < nseg; ++s)
    for (int side = 0; side < 2; ++side) {
      const int i = side ? g2[s] : g1[s];
      const size_t q = (size_t)off[i >> 5] + (i & 31) + 32 * (size_t)fill[i]++;
      sx[q] = (s << 1) | side;
      col[q] = side ? g1[s] : g2[s];
      const int d = col[q] - i;
      if (d < -32768 || d > 32767) fit16 = false;
      dc[q] = (short)d;
    }
  DevGuard g(h->dev);
  void *old[] = {h->d_g1, h->d_g2, h->d_sg_meta, h->d_sg_off, h->d_sg_sx, h->d_sg_col,
                 h->d_sg_dc, h->d_segel, h->d_xa, h->d_xas, h->d_sg_c64, h->d_sg_c32,
                 h->d_sg_ct};
  CK(cudaStreamSynchronize(h->stream));
  for (void *p : old)
    if (p) cudaFree(p);
  h->d_g1 = h->d_g2 = h->d_sg_meta = h->d_sg_off = h->d_sg_sx = h->d_sg_col = nullptr;
  h->d_sg_dc = nullptr;
  h->sg16 = false;
  h->d_segel = nullptr;
  h->d_xa = h->d_xas = h->d_sg_c64 = nullptr;
  h->d_sg_c32 = nullptr;
  h->d_sg_ct = nullptr;
  h->has_segments = 0;
  if (h->sto == 3) h->has_matrix = 0;  // the stored segment matrix belonged to the old numbering
  h->sto = 1;
  int st;
  if ((st = dalloc(&h->d_g1, nseg)) || (st = dalloc(&h->d_g2, nseg)) ||
      (st = dalloc(&h->d_sg_meta, n)) || (st = dalloc(&h->d_sg_off, (size_t)nsl + 1)) ||
      (st = dalloc(&h->d_sg_sx, nslot)) || (st = dalloc(&h->d_sg_col, nslot)) ||
      (st = dalloc(&h->d_segel, nseg)) || (st = dalloc(&h->d_xa, 2 * (size_t)nseg)) ||
      (st = dalloc(&h->d_xas, 2 * (size_t)nseg)) || (st = dalloc(&h->d_sg_c64, nslot)) ||
      (st = dalloc(&h->d_sg_c32, nslot)))
    return st;
  CK(cudaMemcpyAsync(h->d_g1, g1.data(), sizeof(int) * nseg, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_g2, g2.data(), sizeof(int) * nseg, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_sg_meta, meta.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_sg_off, off.data(), sizeof(int) * (nsl + 1), cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_sg_sx, sx.data(), sizeof(int) * nslot, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_sg_col, col.data(), sizeof(int) * nslot, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->d_segel, segel.data(), sizeof(int2) * nseg, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaMemsetAsync(h->d_sg_c64, 0, sizeof(double) * nslot, h->stream));
  CK(cudaMemsetAsync(h->d_sg_c32, 0, sizeof(float) * nslot, h->stream));
  if (fit16) {  // the binary32 kernels read 2-byte offsets instead of the columns
    if ((st = dalloc(&h->d_sg_dc, nslot))) return st;
    CK(cudaMemcpyAsync(h->d_sg_dc, dc.data(), sizeof(short) * nslot, cudaMemcpyHostToDevice,
                       h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  h->sg16 = fit16;
  h->nsg = nseg;
  h->nsg_slots = (long long)nslot;
  h->has_segments = 1;
  return BIEF_OK;
}

static int set_matrix_seg_impl(bief_handle *h, const double *da, const double *xa, char typdia,
                               char typext, bool dev) {
  if (!h || !da) return BIEF_ERR_ARGS;
  if (!h->has_segments) return BIEF_ERR_NO_MATRIX;
  if (typdia_code(typdia) < 0) return BIEF_ERR_ARGS;
  if (typext != 'S' && typext != 'Q' && typext != '0') return BIEF_ERR_ARGS;
  if (typext != '0' && !xa) return BIEF_ERR_ARGS;
  DevGuard g(h->dev);
  const size_t n = (size_t)h->npoin;
  const int nc = typext == 'Q' ? 2 : (typext == 'S' ? 1 : 0);
  const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(h->d_dm, da, sizeof(double) * n, kind, h->stream));
  if (nc) CK(cudaMemcpyAsync(h->d_xa, xa, sizeof(double) * nc * h->nsg, kind, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->typdia = typdia == 'q' ? 'Q' : (typdia == 'i' ? 'I' : typdia);
  h->typext = typext;
  h->has_matrix = 1;
  h->sto = 3;
  h->mat_gen++;
  return BIEF_OK;
}

int bief_set_matrix_seg(bief_handle *h, const double *da, const double *xa, char typdia,
                        char typext) {
  return set_matrix_seg_impl(h, da, xa, typdia, typext, false);
}

int bief_set_matrix_seg_dev(bief_handle *h, const double *da, const double *xa, char typdia,
                            char typext) {
  return set_matrix_seg_impl(h, da, xa, typdia, typext, true);
}

int bief_ebe_to_seg(bief_handle *h, void *stream) {
  if (!h) return BIEF_ERR_ARGS;
  if (!h->has_matrix || !h->has_segments) return BIEF_ERR_NO_MATRIX;
  if (h->sto == 3) return BIEF_OK;
  DevGuard g(h->dev);
  cudaStream_t s = (cudaStream_t)stream;
  const int gs = grid_for(h->nsg, h->nsm);
  if (h->typext == 'S')
    k_assex3<true><<<gs, 256, 0, s>>>(h->nsg, h->nelem, h->nelem, h->d_segel, h->d_g1, h->d_ik,
                                      h->d_xm, h->d_xa);
  else if (h->typext == 'Q')
    k_assex3<false><<<gs, 256, 0, s>>>(h->nsg, h->nelem, h->nelem, h->d_segel, h->d_g1, h->d_ik,
                                       h->d_xm, h->d_xa);
  if (h->typext != '0') h->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  h->sto = 3;
  h->mat_gen++;
  return BIEF_OK;
}

int bief_matrix_storage(bief_handle *h) {
  if (!h) return BIEF_ERR_ARGS;
  if (!h->has_matrix) return BIEF_ERR_NO_MATRIX;
  return h->sto;
}

int bief_last_timing(bief_handle *h, float *solve_ms, float *matvec_ms) {
  if (!h) return BIEF_ERR_ARGS;
  if (h->mv_pending) {
    // bief_matvec_dev returns before its kernel ends: read its events once
    // the stream has passed them
    DevGuard g(h->dev);
    if (cudaEventQuery(h->ev[3]) == cudaSuccess) {
      CK(cudaEventElapsedTime(&h->matvec_ms, h->ev[2], h->ev[3]));
      h->mv_pending = 0;
    }
  }
  if (solve_ms) *solve_ms = h->solve_ms;
  if (matvec_ms) *matvec_ms = h->matvec_ms;
  return BIEF_OK;
}

long long bief_kernel_launches(bief_handle *h) { return h ? h->launches : -1; }

}  // extern "C"
