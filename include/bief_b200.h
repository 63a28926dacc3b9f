/*
 * bief_b200.h -- C ABI of the B200 (sm_100a) implementation of BIEF's
 * element-by-element P1 conjugate-gradient solve and matrix-vector product.
 *
 * The entry points replace, for one mesh of 3-node triangles with EBE
 * storage (STO=1, ELMLIN=ELMCOL=11), the reference subroutines
 *
 *   SOLVE(X,A,B,TB,CFG,INFOGR,MESH,AUX)   sources/utils/bief/solve.f:2-5
 *        with CFG%SLV=1 (GRACJG, gracjg.F:2-5) and CFG%PRECON in
 *        {0,1,2,3,5} (diagonal change of variables, precd1.f:88-158)
 *   MATVEC(OP,X,A,Y,C,MESH,LEGO)           sources/utils/bief/matvec.f:2-5
 *        with OP in 'X=AY', 'X=X+AY', 'X=-AY', 'X=X-AY', 'X=X+CAY',
 *        'X=CAY', 'X=TAY', 'X=-TAY', 'X=X+TAY', 'X=X-TAY', 'X=X+CTAY'
 *        (matvec.f:316-380 -> matvct.f:255-306 -> mv0303.f:117-630)
 *
 * Conventions (those of the Fortran caller):
 *   - IKLE is the Fortran array IKLE(NELMAX,3): column-major, 1-based.
 *   - XM is A%X%R viewed as XM(NELMAX,NDIAG): NDIAG=3 for symmetric storage
 *     TYPEXT='S' (columns M12,M13,M23) or 6 for TYPEXT='Q' (then M21,M31,
 *     M32), following om1111.f:43-50.  DM is A%D%R(NPOIN).
 *   - TYPDIA is 'Q' (any diagonal), 'I' (identity) or '0' (zero).
 *   - Host pointers unless the function name ends in _dev.  The _dev
 *     functions take a cudaStream_t (as void*) and run in stream order on
 *     it; NULL is CUDA's default stream.  The host-pointer functions use the
 *     handle's own stream and return after the results are on the host.
 *   - Every function returns an int status: 0 = success; > 0 = the solve
 *     stopped at NITMAX without converging (the value is the iteration
 *     count); < 0 = an error (see BIEF_ERR_*).  The reference aborts with
 *     PLANTE(1) on errors; a Fortran shim maps < 0 to PLANTE(1).
 *   - A handle owns one CUDA stream and its device buffers; calls on one
 *     handle must not overlap.  Different handles are independent.
 *
 * Floating point: the binary64 solve performs the reference's operations in
 * the reference's order with no fused multiply-add, so the matrix-vector
 * product, the change of variables and every vector update are bit-identical
 * to the Fortran; only the dot products are summed in a fixed parallel tree
 * (bief_launch_info gives its shape).
 */
#ifndef BIEF_B200_H
#define BIEF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define BIEF_OK                   0
#define BIEF_ERR_ARGS            -1  /* bad argument / unknown OP string   */
#define BIEF_ERR_BREAKDOWN       -2  /* D.AD <= 0: matrix not SPD           */
#define BIEF_ERR_NAN             -3  /* NaN/Inf met in the iteration         */
#define BIEF_ERR_BAD_MESH        -4  /* IKLE entry outside 1..NPOIN          */
#define BIEF_ERR_UNSUPPORTED     -5  /* SLV/PRECON/storage not on this path  */
#define BIEF_ERR_CUDA            -6  /* CUDA runtime error                   */
#define BIEF_ERR_DEVICE_TIMEOUT  -7  /* a grid barrier wait ran out          */
#define BIEF_ERR_NO_MATRIX       -8  /* solve/matvec before set_matrix       */
#define BIEF_ERR_SIZE            -9  /* problem larger than a fixed limit    */

/* Mirror of TYPE(SLVCFG) (bief_def.f:506-532). */
typedef struct {
    int    slv;     /* 1 CG, 2 RESCJG, 3 EQUNOR, 4 ERRMIN, 5 CGSQUA, 6 CGSTAB, 7 GMRES */
    int    nitmax;  /* maximum number of iterations                        */
    int    precon;  /* 0/1 none, 2 diagonal, 3 (=2 for one matrix), 5 |diag| */
    int    krylov;  /* unused by CG                                        */
    double eps;     /* relative (or absolute, when ||B||^2 < 1) accuracy    */
    double zero;    /* unused by CG                                        */
    int    ok;      /* out: 1 when the accuracy was reached                */
    int    nit;     /* out: iterations done                                */
} bief_slvcfg;

typedef struct bief_handle bief_handle;

/* Solve flags */
#define BIEF_SOLVE_MUTATE_INPUTS  1  /* leave B = D.B and the stored matrix
                                        = D.A.D (TYPDIA 'I'), as SOLVE does */
#define BIEF_SOLVE_INFOGR         2  /* print the method's iteration message */
#define BIEF_SOLVE_MODASS3        4  /* MODASS = 3: compensated dot products
                                        (dot_comp.f), as P_DOTS switches to
                                        them for every method (p_dots.f:148-
                                        156); fold the RHS error vector B%E
                                        into B first, as SOLVE does
                                        (solve.f:546-549) */

/* Mesh: replaces the MESH%IKLE / NPOIN / NELEM / NELMAX part of BIEF_MESH
 * (bief_def.f:205-498).  Validates IKLE and builds the node->element
 * gather index used instead of ASSVEC's scatter (assvec.f:88-93).  All
 * device memory for the mesh, one matrix and the solver work vectors
 * (SOLVE's TBB blocks, solve.f:192-209) is allocated here, once. */
int bief_mesh_create(int npoin, int nelem, int nelmax, const int *ikle,
                     int device, bief_handle **out);
int bief_destroy(bief_handle *h);

/* Matrix A%D, A%X, A%TYPDIA, A%TYPEXT of a BIEF_OBJ with STO=1
 * (bief_def.f:74-196): host arrays copied to the device. */
int bief_set_matrix(bief_handle *h, const double *dm, const double *xm,
                    char typdia, char typext);
/* Device-array variant: dm[npoin], xm[ndiag*nelem] with leading dim nelem. */
int bief_set_matrix_dev(bief_handle *h, const double *dm, const double *xm,
                        char typdia, char typext);
/* Read back the stored matrix (e.g. after a mutating solve). */
int bief_get_matrix(bief_handle *h, double *dm, double *xm, char *typdia);

/* SOLVE(X,A,B,...) for SLV=1 (GRACJG, gracjg.F), SLV=2 (RESCJG, conjugate
 * residual, rescjg.f), SLV=3 (EQUNOR, CG on the normal equations,
 * equnor.f), SLV=4 (ERRMIN, minimum error, errmin.f), SLV=5 (CGSQUA,
 * conjugate gradient squared, cgsqua.f), SLV=6 (CGSTAB, cgstab.f) and
 * SLV=7 (GMRES(KRYLOV), gmres.f, KRYLOV 1..20, NITMAX counting restarts):
 * host X
 * (initial guess in, solution out)
 * and B.  relres_out receives the relative residual the method prints
 * (SQRT(RMRM/XL), or NR0/NB for GMRES).  Other SLV values return
 * BIEF_ERR_UNSUPPORTED. */
int bief_solve(bief_handle *h, double *x, double *b, bief_slvcfg *cfg,
               int flags, double *relres_out);
/* Same with device pointers, on `stream`. */
int bief_solve_dev(bief_handle *h, double *x, double *b, bief_slvcfg *cfg,
                   int flags, double *relres_out, void *stream);

/* Mixed precision (no reference counterpart): binary32 copy of the scaled
 * operator and one binary32 CG whose correction is folded into the binary64
 * solution (a refinement step: x += z, r = b - A x in binary64, binary32
 * residual restarted from r, search direction kept) each time its residual
 * has dropped by the factor inner_tol since the last refinement (0.1 keeps
 * the iteration count of binary64 CG; smaller values refine less often).
 * Stops when the binary64 residual reaches outer_tol (relative to ||D.B||,
 * absolute when that is < 1).  B is not modified.  outer_out/inner_out:
 * refinement steps and total inner iterations.  Symmetric matrices only;
 * the binary32 operator holds at most 64 neighbours per node (EBE storage),
 * BIEF_ERR_SIZE beyond (the binary64 SOLVE has no such limit). */
int bief_solve_mixed(bief_handle *h, double *x, const double *b,
                     int precon, double inner_tol, double outer_tol,
                     int max_outer, int max_inner, int *outer_out,
                     int *inner_out, double *relres_out);
int bief_solve_mixed_dev(bief_handle *h, double *x, const double *b,
                         int precon, double inner_tol, double outer_tol,
                         int max_outer, int max_inner, int *outer_out,
                         int *inner_out, double *relres_out, void *stream);

/* MATVEC(OP,X,A,Y,C,MESH,LEGO=.TRUE.): OP is the reference's 8-character
 * operation string (trailing blanks optional). */
int bief_matvec(bief_handle *h, const char *op, double *x, const double *y,
                double c);
int bief_matvec_dev(bief_handle *h, const char *op, double *x,
                    const double *y, double c, void *stream);

/* MATVEC 'X=AY' in binary32 (no reference counterpart: the product of the
 * mixed-precision inner CG, on the stored matrix): device X and Y of NPOIN
 * floats, X_i = s_i Y_i + sum_j c_ij (Y_j - Y_i) with binary32 coefficients
 * assembled per neighbour from the EBE (or segment) matrix and s_i the
 * binary32 row sum.  The first call after the matrix changed (or after a
 * mixed solve, which reuses the same buffers) builds that copy; later calls
 * only run the product.  Symmetric matrices only (BIEF_ERR_UNSUPPORTED
 * otherwise).  X may alias Y.  Timing through bief_last_timing. */
int bief_matvec32_dev(bief_handle *h, float *x, const float *y, void *stream);

/* Wave-equation operator A = M + coef_e K_e assembled on the device the way
 * PROPAG assembles AM1 (propag.F:661-677,1407): MT01AA mass (mt01aa.f:82-
 * 103) plus MT02AA P0 diffusion (mt02aa.f:106-149), diagonals assembled by
 * ASSVEC (matrix.f:218-227) and summed by OM 'M=M+N' (om1111.f:299-312).
 * x, y: node coordinates; coef: per-element coefficient (device arrays).
 * Stores the result as the handle's matrix (TYPDIA 'Q', TYPEXT 'S'). */
int bief_assemble_wave_dev(bief_handle *h, const double *x, const double *y,
                           const double *coef, void *stream);

/* The general form of the same assembly, as PROPAG's two MATRIX calls build
 * AM1: 'M=N' MATMAS with XMUL = xmul_mass (propag.F:673-676, mt01aa.f), then
 * 'M=M+N' with the diffusion matrix of XMUL = xmul_dif (propag.F:1407-1408):
 *   kind 10  MATDIF, u per element (P0, mt02aa.f:106-149)
 *   kind 11  MATDIF, u per node (P1, mt02aa.f:244-279)
 *   kind 12  MATDIFUV, u and v per node (mt02aa.f:200-240): PROPAG's own
 *            call, with u = DM1, v = HPROP and XMUL = -1.
 * Device arrays; v is read for kind 12 only.  Stores the result as the
 * handle's matrix (TYPDIA 'Q', TYPEXT 'S'). */
int bief_assemble_mass_diff_dev(bief_handle *h, const double *x, const double *y,
                                double xmul_mass, double xmul_dif, int kind,
                                const double *u, const double *v, void *stream);
/* Copy the stored matrix to device arrays dm[npoin] and xm: EBE storage
 * xm[ndiag*nelem] (leading dimension NELEM), segment storage xa[ncol*nseg]. */
int bief_get_matrix_dev(bief_handle *h, double *dm, double *xm, void *stream);

/* ---- Segment (edge) storage, MATRIX STORAGE = 3 ------------------------
 * The segment numbering of the mesh: MESH%GLOSEG(MAXSEG,2) as STOSEG builds
 * it (stoseg.f:94-225), 1-based, column-major, nseg <= maxseg segments.
 * Every element face must be exactly one segment (the element-to-segment
 * map that ASSEX3 uses is derived from it).  Replaces an earlier numbering;
 * a stored segment matrix is dropped with it.  Replaces no reference
 * routine: the Fortran side passes its MESH%GLOSEG once per mesh. */
int bief_set_segments(bief_handle *h, int nseg, int maxseg, const int *gloseg);
/* Matrix in segment storage (STO=3): DA(NPOIN) and XA(NSEG) for TYPEXT
 * 'S' or XA(NSEG,2) for 'Q' (column 1: the coefficient of row GLOSEG(,1),
 * column 2: of row GLOSEG(,2)).  bief_matvec then follows MVSEG
 * (mvseg.f:110-720, via matvct.f:665-689), bief_solve / bief_solve_mixed
 * scale it with OMSEG 'M=DMD' (omseg.f:509-541) and iterate on it. */
int bief_set_matrix_seg(bief_handle *h, const double *da, const double *xa,
                        char typdia, char typext);
int bief_set_matrix_seg_dev(bief_handle *h, const double *da,
                            const double *xa, char typdia, char typext);
/* ASSEX3 (assex3.f:150-160 -> as3_1111_s.f / as3_1111_q.f): the stored EBE
 * matrix becomes segment storage (off-diagonal terms summed per segment in
 * element order; the diagonal unchanged).  Needs bief_set_segments. */
int bief_ebe_to_seg(bief_handle *h, void *stream);
/* Storage of the stored matrix: 1 (EBE) or 3 (segments). */
int bief_matrix_storage(bief_handle *h);

/* Adjoint gradient of a loss through x = A(coef)^-1 b with
 * A = M + coef_e K_e: grad[e] = -lambda_e^T K_e x_e (K_e from MT02AA with
 * unit coefficient), for device arrays lambda[npoin], x[npoin],
 * x/y coordinates; writes grad[nelem].  No reference counterpart. */
int bief_wave_coef_grad_dev(bief_handle *h, const double *xc,
                            const double *yc, const double *lambda,
                            const double *x, double *grad, void *stream);

/* Adjoint gradient through x = A(u, v)^-1 b with A assembled by
 * bief_assemble_mass_diff_dev (kind 11: MATDIF with u per node; kind 12:
 * MATDIFUV with u and v per node, PROPAG's form with u = DM1 and v = HPROP,
 * the depth): given lambda with A^T lambda = dL/dx, writes
 * gu[i] = dL/du_i (npoin) and, for kind 12, gv[i] = dL/dv_i, summed per
 * node over its elements without atomics.  xmul_dif is the diffusion
 * matrix's XMUL.  Device arrays.  No reference counterpart. */
int bief_mass_diff_grad_dev(bief_handle *h, const double *xc, const double *yc,
                            double xmul_dif, int kind, const double *u, const double *v,
                            const double *lambda, const double *x, double *gu, double *gv,
                            void *stream);

/* Batched mixed-precision solve (no reference counterpart): the handle's
 * mesh is block diagonal with ninst <= 512 independent instances, instance
 * i owning nodes [node_off[i], node_off[i]+npoin_inst[i]) (node_off[i] a
 * multiple of 32, no element coupling two instances).  All instances run
 * the bief_solve_mixed algorithm in ONE persistent launch, each with its own
 * scalars and convergence mask; nodes_per_thread (1, 2, 4, 8) and
 * threads_per_block (256, 512 or 1024; 0 means 1024) set the work tile
 * (threads_per_block*nodes_per_thread nodes), the block shape and the
 * per-instance dot order.  x, b:
 * device arrays over the whole mesh; per-instance results in host arrays
 * status (0 / inner iterations when not converged / < 0 error), outer_out,
 * inner_out, relres_out.  Either storage: with segment storage (STO=3)
 * the segment numbering set by bief_set_segments holds every instance's
 * segments, each instance's in its own order. */
int bief_batch_solve_mixed_dev(bief_handle *h, int ninst, const int *node_off,
                               const int *npoin_inst, double *x, const double *b,
                               int precon, double inner_tol, double outer_tol,
                               int max_outer, int max_inner,
                               int nodes_per_thread, int threads_per_block, int *status,
                               int *outer_out, int *inner_out,
                               double *relres_out, void *stream);

/* DIRI01 (diri01.f:90-130 with DIRAUX, diraux.f:70-85) for Dirichlet values
 * on the NPTFR boundary points: nbor = MESH%NBOR (1-based), limdir = LIMDIR,
 * points with limdir[k] == kdir get the value fbor[k].  SM (npoin) becomes
 * SM - A W1 (W1 = the Dirichlet values) with SM = D*FBOR and F = FBOR at the
 * Dirichlet points; with maskpt (npoin, or NULL) SM and F are masked; the
 * stored matrix keeps its diagonal and loses the off-diagonal terms of the
 * Dirichlet rows and columns (OM 'M=DMD'), in either storage.  Host arrays;
 * the _dev variant takes device arrays and runs on `stream`, which it
 * synchronises when nptfr > 0 to report an NBOR entry outside 1..NPOIN
 * (BIEF_ERR_BAD_MESH; such entries are skipped, never written through). */
int bief_diri01(bief_handle *h, int nptfr, const int *nbor, const int *limdir,
                int kdir, const double *fbor, double *sm, double *f,
                const double *maskpt);
int bief_diri01_dev(bief_handle *h, int nptfr, const int *nbor,
                    const int *limdir, int kdir, const double *fbor, double *sm,
                    double *f, const double *maskpt, void *stream);

/* Self-test of the device-side bounded waits (no reference counterpart):
 * runs one block into a grid barrier that can never complete and checks that
 * its wait gives up after timeout_ns (1e6..5e9) with a recorded timeout.
 * Returns BIEF_ERR_DEVICE_TIMEOUT when the wait ended as designed (the
 * device stays usable), another status otherwise.  The solvers use the same
 * wait with a 2 s limit. */
int bief_selftest_timeout(int device, long long timeout_ns);

/* Shape of the device dot-product tree: number of blocks and threads per
 * block of the persistent solver kernel. */
int bief_launch_info(bief_handle *h, int *nblocks, int *nthreads);
/* Residency of the persistent solver kernels: 1 = one block per SM (every
 * register to one 1024-thread block), 2 = two blocks per SM (half the
 * registers each, twice the warps to hide memory latency: faster once a
 * solve streams its operator from HBM, slower while it stays in L2),
 * 0 = automatic, the choice bief_mesh_create makes: two when the binary32
 * operator and vectors (about 80 B per node) exceed 2.25 times the L2 cache
 * (about 3.5M nodes on a B200, where the two measure the same).  It sets
 * the shape of the dot-product tree (bief_launch_info) and so the bits of
 * the dot products; the batched solver takes it too (its dot order does not
 * depend on it). */
int bief_set_blocks_per_sm(bief_handle *h, int blocks_per_sm);
/* Which gather records the standalone MATVEC (bief_matvec*) reads for this
 * mesh, fixed when the mesh is made: the most compact its numbering allows.
 * The bits of the product are the same in every format. */
#define BIEF_MV_IKLE   0  /* a node in more than 255 elements: element index, then IKLE */
#define BIEF_MV_LOCAL  1  /* 16-bit element offsets and vertex offsets: 6 B per entry  */
#define BIEF_MV_BAND   2  /* element index, 16-bit vertex offsets: 8 B per entry       */
#define BIEF_MV_ANY    3  /* element index and both other vertices: 12 B per entry     */
int bief_matvec_format(bief_handle *h, int *format);
/* Kernel time (ms, CUDA events recorded around the launch on the stream
 * the call used) of the last solve kernel and of the last matvec kernel.  For
 * bief_matvec_dev, which returns before its kernel ends, the matvec time is
 * that of the last call whose kernel had completed when this is called. */
int bief_last_timing(bief_handle *h, float *solve_ms, float *matvec_ms);
/* Number of device kernels the library launched since the handle was made. */
long long bief_kernel_launches(bief_handle *h);

const char *bief_strerror(int status);

/* SOLVE (SLV=1, diagonal preconditioning) for callers that cannot allocate
 * device memory, e.g. a host code whose device arrays are owned by an
 * OpenACC/OpenMP data region or a pool allocator, or that must not call
 * cudaMalloc/cudaFree (and their implicit synchronisation) inside its time
 * loop.  No counterpart in the reference: it is the same GRACJG as
 * bief_solve_dev, but takes no handle and allocates nothing.  All arrays
 * are the caller's device arrays: IKLE(NELMAX,3) 1-based, DM(NPOIN),
 * XM(NELMAX,NDIAG), X, B.  As the reference SOLVE does, it leaves
 * B = D.B, DM and XM = the scaled D.A.D (TYPDIA 'I' for PRECON 2/3).
 * Everything else (gather index, work vectors, reduction partials) lives
 * in one fixed ~6.6 MB device array inside the library: at most 65,536
 * nodes and 131,072 elements (NELMAX), else BIEF_ERR_SIZE.  Calls share
 * that array, so calls that overlap on the GPU race; the first call on a
 * device looks up the array's address and should come before any stream
 * capture.  Every call, not only the first, waits for its stream twice
 * (the IKLE check and the result are read back to the host before it
 * returns).  Configuration errors get bief_solve's codes; SLV other than 1
 * is BIEF_ERR_UNSUPPORTED.  TYPEXT 'S' or 'Q'. */
int bief_solve_noalloc(int npoin, int nelem, int nelmax, const int *ikle,
                       double *dm, double *xm, char typdia, char typext,
                       double *x, double *b, bief_slvcfg *cfg,
                       double *relres_out, int device, void *stream);

#ifdef __cplusplus
}
#endif
#endif
