/*
 * bief_oracle.h -- CPU restatement of TELEMAC-MASCARET BIEF's EBE P1
 * conjugate-gradient path (SOLVE -> PRECD1 -> GRACJG -> MATVEC/MV0303 +
 * ASSVEC), written in plain C for use as a TEST ORACLE ONLY.
 *
 * This code is test infrastructure: only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark may load it.  The product library never
 * links it and never falls back to it.
 *
 * Parity status: UNPINNED by the reference itself.  The reference is Fortran
 * and no Fortran compiler is available, and the reference ships no
 * solver-level golden vectors.  The restatement is cross-checked instead
 * against an independent dense/scipy computation (tests/test_oracle.py).
 *
 * Conventions: 0-based node numbers; connectivity as three columns
 * ik0/ik1/ik2 (the reference's IKLE(NELMAX,3) columns); off-diagonal
 * element terms as structure-of-arrays columns of length `ld`
 * (XM(IELEM,1..3) = M12,M13,M23 for symmetric 'S' storage, plus
 * M21,M31,M32 for 'Q' storage, following om1111.f's convention).
 * All arithmetic is IEEE binary64 with no fused multiply-add contraction
 * (compile with -ffp-contract=off), matching an x86-64 build of the
 * reference with its default flags.
 */
#ifndef BIEF_ORACLE_H
#define BIEF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* dot-product summation orders */
#define ORC_DOT_SEQUENTIAL 0 /* dot.f:53, the reference's left-to-right sum */
#define ORC_DOT_BLOCKED    1 /* the device kernels' fixed block/tree order   */
#define ORC_DOT_COMP_SEQUENTIAL 2 /* MODASS=3: dot_comp.f (Dot2), sequential  */
#define ORC_DOT_COMP_BLOCKED    3 /* MODASS=3 in the device kernels' order      */

/* status codes (identical values to the product library's) */
#define ORC_OK             0
#define ORC_ERR_ARGS      -1
#define ORC_ERR_BREAKDOWN -2
#define ORC_ERR_NAN       -3
#define ORC_ERR_BAD_MESH  -4
#define ORC_ERR_UNSUPPORTED -5

/* Host threads for large checks (default 1: the sequential code).  Only
 * loops with independent iterations are shared out; results are the same
 * bits with any count. */
void orc_set_threads(int n);

int orc_geometry(int nelem, const double *x, const double *y,
                 const int *ik0, const int *ik1, const int *ik2,
                 double *xel2, double *xel3, double *yel2, double *yel3,
                 double *surfac);

void orc_mt01aa(int nelem, double xmul, const double *surfac,
                double *a11, double *a12, double *a13,
                double *a22, double *a23, double *a33);

void orc_mt02aa_p0(int nelem, double xmul, const double *u,
                   const double *xel2, const double *xel3,
                   const double *yel2, const double *yel3,
                   const double *surfac,
                   double *a11, double *a12, double *a13,
                   double *a22, double *a23, double *a33);

void orc_assvec(double *x, int npoin, int nelem,
                const int *ik0, const int *ik1, const int *ik2,
                const double *w1, const double *w2, const double *w3,
                int init);

int orc_wave_matrix(int npoin, int nelem, const double *x, const double *y,
                    const int *ik0, const int *ik1, const int *ik2,
                    const double *coef, double *dm, double *xm);

void orc_mt02aa_p1(int nelem, double xmul, const double *u,
                   const int *ik0, const int *ik1, const int *ik2,
                   const double *xel2, const double *xel3,
                   const double *yel2, const double *yel3,
                   const double *surfac,
                   double *a11, double *a12, double *a13,
                   double *a22, double *a23, double *a33);

void orc_mt02aa_uv(int nelem, double xmul, const double *u, const double *v,
                   const int *ik0, const int *ik1, const int *ik2,
                   const double *xel2, const double *xel3,
                   const double *yel2, const double *yel3,
                   const double *surfac,
                   double *a11, double *a12, double *a13,
                   double *a22, double *a23, double *a33);

int orc_mass_diff_matrix(int npoin, int nelem, const double *x, const double *y,
                         const int *ik0, const int *ik1, const int *ik2,
                         double xmul_mass, double xmul_dif, int kind,
                         const double *u, const double *v, double *dm, double *xm);

int orc_wave_matrix_parts(int npoin, int nelem, const double *x, const double *y,
                          const int *ik0, const int *ik1, const int *ik2,
                          double *kxm);

int orc_matvec(const char *op, int npoin, int nelem,
               const int *ik0, const int *ik1, const int *ik2,
               double *x, const double *da, char typdia,
               const double *xm, int ld, char typext,
               const double *y, double c, double *t, double *w);

double orc_dot(int n, const double *x, const double *y);
double orc_dot_blocked(int n, const double *x, const double *y,
                       int nblocks, int nthreads);
double orc_dot_comp(int n, const double *x, const double *y);
double orc_dot_blocked_comp(int n, const double *x, const double *y,
                            int nblocks, int nthreads);

int orc_precd1(int npoin, int nelem, const int *ik0, const int *ik1,
               const int *ik2, int precon, double *x, double *dm,
               char *typdia, double *xm, int ld, char typext, double *b,
               double *d);

int orc_gracjg(int npoin, int nelem, const int *ik0, const int *ik1,
               const int *ik2, double *x, const double *da, char typdia,
               const double *xm, int ld, char typext, const double *b,
               int nitmax, double eps, int dot_mode, int nblocks,
               int nthreads, int *nit_out, double *relres_out,
               int *relat_out);

int orc_solve(int npoin, int nelem, const int *ik0, const int *ik1,
              const int *ik2, double *x, double *b, double *dm,
              char *typdia, double *xm, int ld, char typext, int slv,
              int precon, int nitmax, double eps, int dot_mode,
              int nblocks, int nthreads, int *nit_out, double *relres_out,
              int *relat_out, int krylov);

int orc_solve_mixed(int npoin, int nelem, const int *ik0, const int *ik1,
                    const int *ik2, double *x, const double *b,
                    const double *dm, char typdia, const double *xm,
                    char typext, int precon, double inner_tol,
                    double outer_tol, int max_outer, int max_inner,
                    int nblocks, int nthreads, int *outer_out,
                    int *inner_total_out, double *relres_out);

double orc_dot_batch(int n, const double *x, const double *y, int nt, int npt);

int orc_solve_mixed_batch(int npoin, int nelem, const int *ik0, const int *ik1,
                          const int *ik2, double *x, const double *b,
                          const double *dm_in, char typdia_in, const double *xm_in,
                          char typext, int precon, double inner_tol,
                          double outer_tol, int max_outer, int max_inner,
                          int nt, int npt, int *outer_out, int *inner_total_out,
                          double *relres_out);
int orc_solve_mixed_batch_seg(int npoin, int nseg, const int *g1, const int *g2, double *x,
                              const double *b, const double *dm_in, char typdia_in,
                              const double *xa_in, char typext, int precon, double inner_tol,
                              double outer_tol, int max_outer, int max_inner, int nt, int npt,
                              int *outer_out, int *inner_total_out, double *relres_out);

int orc_solve_omp(int npoin, int nelem, const int *ik0, const int *ik1,
                  const int *ik2, double *x, const double *b_in,
                  const double *dm_in, const double *xm_in, int nitmax,
                  double eps, int nthreads, int *nit_out, double *relres_out);

/* segment storage (STO=3): 0-based GLOSEG columns g1/g2; ELTSEG/ORISEG as
 * 3 x nelem face-major arrays */
int orc_stoseg(int npoin, int nelem, const int *ik0, const int *ik1, const int *ik2,
               int neleb, const int *nelbor, const int *nulone, int *g1, int *g2,
               int *eltseg, int *oriseg, int *nseg_out);

int orc_assex3(int nelem, const int *eltseg, const int *oriseg, char typext,
               const double *xmt, int ld, int nseg, double *xa);

int orc_mvseg(const char *op, int npoin, int nseg, const int *g1, const int *g2,
              double *x, const double *da, char typdia, const double *xa,
              char typext, const double *y, double c);

int orc_solve_seg(int npoin, int nseg, const int *g1, const int *g2, double *x, double *b,
                  double *dm, char *typdia, double *xa, char typext, int slv, int precon,
                  int nitmax, double eps, int dot_mode, int nb, int nt, int *nit_out,
                  double *relres_out, int *relat_out, int krylov);

int orc_solve_mixed_seg(int npoin, int nseg, const int *g1, const int *g2, double *x,
                        const double *b, const double *dm_in, char typdia_in,
                        const double *xa_in, char typext, int precon, double inner_tol,
                        double outer_tol, int max_outer, int max_inner, int nb, int nt,
                        int *outer_out, int *inner_total_out, double *relres_out);

/* DIRI01 with boundary values (0-based nbor); xm/xa, sm and f modified */
int orc_diri01(int npoin, int nelem, const int *ik0, const int *ik1, const int *ik2,
               const double *dm, char typdia, double *xm, char typext, int nptfr,
               const int *nbor, const int *limdir, int kdir, const double *fbor, double *sm,
               double *f, const double *maskpt);
int orc_diri01_seg(int npoin, int nseg, const int *g1, const int *g2, const double *dm,
                   char typdia, double *xa, char typext, int nptfr, const int *nbor,
                   const int *limdir, int kdir, const double *fbor, double *sm, double *f,
                   const double *maskpt);

#ifdef __cplusplus
}
#endif
#endif
