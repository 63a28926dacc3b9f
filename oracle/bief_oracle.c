/*
 * bief_oracle.c -- CPU restatement of BIEF's EBE P1 CG path.  TEST ORACLE
 * ONLY (see bief_oracle.h): loaded by the tests, the smoke check and the
 * benchmark's CPU-baseline leg, never by the product library.
 *
 * Parity unpinned: the Fortran reference cannot be compiled here and ships
 * no solver-level golden vectors; see tests/test_oracle.py for the
 * independent dense/scipy cross-checks that stand in for a pin.
 *
 * Every routine names the reference lines it restates (paths relative to
 * the TELEMAC-MASCARET source tree).  Loop orders and operand orders are
 * kept as in the Fortran so that the binary64 results are the same bits an
 * x86-64 build of the reference produces (no FMA contraction).
 */
#include "bief_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Host threads for the large-case checks (orc_set_threads).  With 1, the
 * default, every routine runs the sequential code below.  With more, the
 * loops whose iterations are independent (vector updates, per-node
 * gathers, per-block dot partials) are shared out with OpenMP; each
 * iteration computes exactly what it computes sequentially and every sum
 * keeps its order, so the results are the same bits (checked by
 * tests/test_oracle_threads.py). */
static int orc_nthreads = 1;

void orc_set_threads(int n)
{
    orc_nthreads = n < 1 ? 1 : n;
}

/* Whether a loop of n iterations is shared out. */
#define ORC_PAR(n) (orc_nthreads > 1 && (long long)(n) >= 4096)
#define ORC_MAX_NT 1024
#define ORC_PRAGMA(x) _Pragma(#x)
/* a vector loop of n independent iterations */
#define ORC_PFOR(n) ORC_PRAGMA(omp parallel for if (ORC_PAR(n)) num_threads(orc_nthreads) schedule(static))

/* ------------------------------------------------------------------ */
/* mesh geometry                                                        */
/* ------------------------------------------------------------------ */

/* inbief.f:369-391 -- XEL/YEL relative to the element's first node
 * (OV_2 'X=X-Y   '), surv11.f:56-64 -- SURFAC = 0.5*(X2*Y3-X3*Y2),
 * geoelt.f:73-84 -- a determinant below 1e-20 is a fatal mesh error. */
int orc_geometry(int nelem, const double *x, const double *y,
                 const int *ik0, const int *ik1, const int *ik2,
                 double *xel2, double *xel3, double *yel2, double *yel3,
                 double *surfac)
{
    for (int e = 0; e < nelem; ++e) {
        double x1 = x[ik0[e]], y1 = y[ik0[e]];
        double X2 = x[ik1[e]] - x1;
        double X3 = x[ik2[e]] - x1;
        double Y2 = y[ik1[e]] - y1;
        double Y3 = y[ik2[e]] - y1;
        xel2[e] = X2; xel3[e] = X3; yel2[e] = Y2; yel3[e] = Y3;
        surfac[e] = 0.5 * (X2 * Y3 - X3 * Y2);
        double det = X2 * Y3 - Y2 * X3; /* geoelt.f:80 T12*T23-T22*T13 */
        if (det < 1.0e-20) return ORC_ERR_BAD_MESH;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* element matrices                                                     */
/* ------------------------------------------------------------------ */

/* mt01aa.f:82-103 -- P1 mass matrix: off-diagonals S/12*XMUL, diagonal
 * twice that (DET + DET). */
void orc_mt01aa(int nelem, double xmul, const double *surfac,
                double *a11, double *a12, double *a13,
                double *a22, double *a23, double *a33)
{
    double sur12 = xmul / 12.0;
    for (int e = 0; e < nelem; ++e) {
        double det = surfac[e] * sur12;
        a12[e] = det; a13[e] = det; a23[e] = det;
        a11[e] = det + det; a22[e] = det + det; a33[e] = det + det;
    }
}

/* mt02aa.f:106-149 -- P1 diffusion matrix with a P0 (per-element)
 * isotropic coefficient U (IELMNU=10, ISO=1). */
void orc_mt02aa_p0(int nelem, double xmul, const double *u,
                   const double *xel2, const double *xel3,
                   const double *yel2, const double *yel3,
                   const double *surfac,
                   double *a11, double *a12, double *a13,
                   double *a22, double *a23, double *a33)
{
    for (int e = 0; e < nelem; ++e) {
        double X2 = xel2[e], X3 = xel3[e], Y2 = yel2[e], Y3 = yel3[e];
        double s2d = xmul * 0.25 / surfac[e];
        double visc1 = u[e] * s2d;
        double bpe = visc1 * (Y3 * Y3 + X3 * X3);
        double cpf = visc1 * (Y2 * Y3 + X2 * X3);
        double apd = visc1 * (Y2 * Y2 + X2 * X2);
        a11[e] = apd + bpe - 2.0 * cpf;
        a22[e] = bpe;
        a33[e] = apd;
        a12[e] = cpf - bpe;
        a13[e] = cpf - apd;
        a23[e] = -cpf;
    }
}

/* assvec.f:80-93 + assve1.f:101 (MODASS=1, LV=1, no mask): X(IKLE(E,IDP))
 * += W(E,IDP), local point IDP outer, element inner. */
void orc_assvec(double *x, int npoin, int nelem,
                const int *ik0, const int *ik1, const int *ik2,
                const double *w1, const double *w2, const double *w3,
                int init)
{
    if (init) for (int i = 0; i < npoin; ++i) x[i] = 0.0;
    const int *ik[3] = {ik0, ik1, ik2};
    const double *w[3] = {w1, w2, w3};
    for (int idp = 0; idp < 3; ++idp)
        for (int e = 0; e < nelem; ++e)
            x[ik[idp][e]] = x[ik[idp][e]] + w[idp][e];
}

/* The wave-equation operator A = M + coef_e * K_e built the way PROPAG
 * builds AM1: MATRIX('M=N', mass) then MATRIX('M=M+N', diffusion)
 * (propag.F:661-677,1407).  Each MATRIX call assembles its own diagonal
 * with ASSVEC (matrix.f:218-227) and OM1111 'M=M+N' adds diagonals and
 * off-diagonals with OV 'X=X+Y' (om1111.f:299-312).  The mass term uses
 * XMUL=1; the diffusion term uses XMUL=1 and U(e)=coef[e].
 * Output: dm[npoin], xm[3*nelem] (columns M12, M13, M23). */
int orc_wave_matrix(int npoin, int nelem, const double *x, const double *y,
                    const int *ik0, const int *ik1, const int *ik2,
                    const double *coef, double *dm, double *xm)
{
    double *g = (double *)malloc(sizeof(double) * 5 * (size_t)nelem);
    double *a = (double *)malloc(sizeof(double) * 6 * (size_t)nelem);
    double *dn = (double *)malloc(sizeof(double) * (size_t)npoin);
    if (!g || !a || !dn) { free(g); free(a); free(dn); return ORC_ERR_ARGS; }
    double *xel2 = g, *xel3 = g + nelem, *yel2 = g + 2 * (size_t)nelem,
           *yel3 = g + 3 * (size_t)nelem, *surf = g + 4 * (size_t)nelem;
    int st = orc_geometry(nelem, x, y, ik0, ik1, ik2, xel2, xel3, yel2, yel3,
                          surf);
    if (st) { free(g); free(a); free(dn); return st; }
    double *a11 = a, *a12 = a + nelem, *a13 = a + 2 * (size_t)nelem,
           *a22 = a + 3 * (size_t)nelem, *a23 = a + 4 * (size_t)nelem,
           *a33 = a + 5 * (size_t)nelem;
    /* mass: M=N */
    orc_mt01aa(nelem, 1.0, surf, a11, a12, a13, a22, a23, a33);
    orc_assvec(dm, npoin, nelem, ik0, ik1, ik2, a11, a22, a33, 1);
    for (int e = 0; e < nelem; ++e) {
        xm[e] = a12[e];
        xm[nelem + e] = a13[e];
        xm[2 * (size_t)nelem + e] = a23[e];
    }
    /* diffusion: M=M+N */
    orc_mt02aa_p0(nelem, 1.0, coef, xel2, xel3, yel2, yel3, surf,
                  a11, a12, a13, a22, a23, a33);
    orc_assvec(dn, npoin, nelem, ik0, ik1, ik2, a11, a22, a33, 1);
    for (int i = 0; i < npoin; ++i) dm[i] = dm[i] + dn[i];
    for (int e = 0; e < nelem; ++e) {
        xm[e] = xm[e] + a12[e];
        xm[nelem + e] = xm[nelem + e] + a13[e];
        xm[2 * (size_t)nelem + e] = xm[2 * (size_t)nelem + e] + a23[e];
    }
    free(g); free(a); free(dn);
    return ORC_OK;
}

/* mt02aa.f:244-279: MATDIF with a P1 viscosity U (one value per node),
 * isotropic:  SOMVX = (U1+U2+U3) XMUL/12 / SURFAC; A12 = -SOMVX X3AUX,
 * A13 = SOMVX X2AUX, A23 = -SOMVX X2X3; diagonals minus the row's others. */
void orc_mt02aa_p1(int nelem, double xmul, const double *u,
                   const int *ik0, const int *ik1, const int *ik2,
                   const double *xel2, const double *xel3,
                   const double *yel2, const double *yel3,
                   const double *surfac,
                   double *a11, double *a12, double *a13,
                   double *a22, double *a23, double *a33)
{
    const double xsur12 = xmul / 12.0;
    for (int e = 0; e < nelem; ++e) {
        double X2 = xel2[e], X3 = xel3[e], Y2 = yel2[e], Y3 = yel3[e];
        double somvx = (u[ik0[e]] + u[ik1[e]] + u[ik2[e]]) * xsur12 / surfac[e];
        double x2x3 = X2 * X3 + Y2 * Y3;
        double x2aux = X2 * (-X2 + X3) + Y2 * (-Y2 + Y3);
        double x3aux = X3 * (-X2 + X3) + Y3 * (-Y2 + Y3);
        a12[e] = -(somvx * x3aux);
        a13[e] = somvx * x2aux;
        a23[e] = -(somvx * x2x3);
        a11[e] = -a12[e] - a13[e];
        a22[e] = -a12[e] - a23[e];
        a33[e] = -a13[e] - a23[e];
    }
}

/* mt02aa.f:200-240: MATDIFUV, U and V both P1:  COEF1 = XMUL/48 / SURFAC;
 * G123 = V1+V2+V3; COEF2 = sum_k U_k (V_k + G123); off-diagonal terms
 * geometry * COEF2 * COEF1; diagonals minus the row's others.  PROPAG adds
 * this to the mass matrix with U = DM1, V = HPROP, XMUL = -1
 * (propag.F:1407-1408). */
void orc_mt02aa_uv(int nelem, double xmul, const double *u, const double *v,
                   const int *ik0, const int *ik1, const int *ik2,
                   const double *xel2, const double *xel3,
                   const double *yel2, const double *yel3,
                   const double *surfac,
                   double *a11, double *a12, double *a13,
                   double *a22, double *a23, double *a33)
{
    const double xsur48 = xmul / 48.0;
    for (int e = 0; e < nelem; ++e) {
        double X2 = xel2[e], X3 = xel3[e], Y2 = yel2[e], Y3 = yel3[e];
        int i1 = ik0[e], i2 = ik1[e], i3 = ik2[e];
        double g1 = v[i1], g2 = v[i2], g3 = v[i3];
        double coef1 = xsur48 / surfac[e];
        double g123 = g1 + g2 + g3;
        double coef2 = u[i1] * (g1 + g123) + u[i2] * (g2 + g123) + u[i3] * (g3 + g123);
        a12[e] = (Y3 * (Y2 - Y3) + X3 * (X2 - X3)) * coef2 * coef1;
        a13[e] = -((Y2 * (Y2 - Y3) + X2 * (X2 - X3)) * coef2 * coef1);
        a23[e] = -((Y2 * Y3 + X2 * X3) * coef2 * coef1);
        a11[e] = -a12[e] - a13[e];
        a22[e] = -a12[e] - a23[e];
        a33[e] = -a13[e] - a23[e];
    }
}

/* AM1 as PROPAG builds it (propag.F:673-676 then :1407-1408): MATRIX
 * 'M=N' MATMAS with XMUL = xmul_mass, then 'M=M+N' with the diffusion
 * matrix of XMUL = xmul_dif; kind 10: MATDIF with U per element
 * (mt02aa.f:106-149), 11: MATDIF with U per node (:244-279), 12: MATDIFUV
 * with U and V per node (:200-240).  Diagonals by ASSVEC per matrix, then
 * OM 'M=M+N' (D and XM added term by term). */
int orc_mass_diff_matrix(int npoin, int nelem, const double *x, const double *y,
                         const int *ik0, const int *ik1, const int *ik2,
                         double xmul_mass, double xmul_dif, int kind,
                         const double *u, const double *v, double *dm, double *xm)
{
    if (kind != 10 && kind != 11 && kind != 12) return ORC_ERR_ARGS;
    if (kind == 12 && !v) return ORC_ERR_ARGS;
    double *g = (double *)malloc(sizeof(double) * 5 * (size_t)nelem);
    double *a = (double *)malloc(sizeof(double) * 6 * (size_t)nelem);
    double *dn = (double *)malloc(sizeof(double) * (size_t)npoin);
    if (!g || !a || !dn) { free(g); free(a); free(dn); return ORC_ERR_ARGS; }
    double *xel2 = g, *xel3 = g + nelem, *yel2 = g + 2 * (size_t)nelem,
           *yel3 = g + 3 * (size_t)nelem, *surf = g + 4 * (size_t)nelem;
    int st = orc_geometry(nelem, x, y, ik0, ik1, ik2, xel2, xel3, yel2, yel3,
                          surf);
    if (st) { free(g); free(a); free(dn); return st; }
    double *a11 = a, *a12 = a + nelem, *a13 = a + 2 * (size_t)nelem,
           *a22 = a + 3 * (size_t)nelem, *a23 = a + 4 * (size_t)nelem,
           *a33 = a + 5 * (size_t)nelem;
    orc_mt01aa(nelem, xmul_mass, surf, a11, a12, a13, a22, a23, a33);
    orc_assvec(dm, npoin, nelem, ik0, ik1, ik2, a11, a22, a33, 1);
    for (int e = 0; e < nelem; ++e) {
        xm[e] = a12[e];
        xm[nelem + e] = a13[e];
        xm[2 * (size_t)nelem + e] = a23[e];
    }
    if (kind == 10)
        orc_mt02aa_p0(nelem, xmul_dif, u, xel2, xel3, yel2, yel3, surf,
                      a11, a12, a13, a22, a23, a33);
    else if (kind == 11)
        orc_mt02aa_p1(nelem, xmul_dif, u, ik0, ik1, ik2, xel2, xel3, yel2, yel3, surf,
                      a11, a12, a13, a22, a23, a33);
    else
        orc_mt02aa_uv(nelem, xmul_dif, u, v, ik0, ik1, ik2, xel2, xel3, yel2, yel3, surf,
                      a11, a12, a13, a22, a23, a33);
    orc_assvec(dn, npoin, nelem, ik0, ik1, ik2, a11, a22, a33, 1);
    for (int i = 0; i < npoin; ++i) dm[i] = dm[i] + dn[i];
    for (int e = 0; e < nelem; ++e) {
        xm[e] = xm[e] + a12[e];
        xm[nelem + e] = xm[nelem + e] + a13[e];
        xm[2 * (size_t)nelem + e] = xm[2 * (size_t)nelem + e] + a23[e];
    }
    free(g); free(a); free(dn);
    return ORC_OK;
}

/* Off-diagonal terms of the unit-coefficient diffusion matrix K_e
 * (mt02aa.f:106-149 with XMUL=1, U=1): kxm[3*nelem] = K12, K13, K23.
 * Used by the adjoint gradient checks. */
int orc_wave_matrix_parts(int npoin, int nelem, const double *x, const double *y,
                          const int *ik0, const int *ik1, const int *ik2,
                          double *kxm)
{
    (void)npoin;
    double *g = (double *)malloc(sizeof(double) * 5 * (size_t)nelem);
    double *a = (double *)malloc(sizeof(double) * 4 * (size_t)nelem);
    double *one = (double *)malloc(sizeof(double) * (size_t)nelem);
    if (!g || !a || !one) { free(g); free(a); free(one); return ORC_ERR_ARGS; }
    for (int e = 0; e < nelem; ++e) one[e] = 1.0;
    double *xel2 = g, *xel3 = g + nelem, *yel2 = g + 2 * (size_t)nelem,
           *yel3 = g + 3 * (size_t)nelem, *surf = g + 4 * (size_t)nelem;
    int st = orc_geometry(nelem, x, y, ik0, ik1, ik2, xel2, xel3, yel2, yel3,
                          surf);
    if (st == ORC_OK)
        orc_mt02aa_p0(nelem, 1.0, one, xel2, xel3, yel2, yel3, surf,
                      a, kxm, kxm + nelem, a + nelem, kxm + 2 * (size_t)nelem,
                      a + 2 * (size_t)nelem);
    free(g); free(a); free(one);
    return st;
}

/* ------------------------------------------------------------------ */
/* matrix-vector product                                                */
/* ------------------------------------------------------------------ */

/* MATVEC 'X=...AY' for an EBE P1-P1 matrix: MATVCT selects MV0303 with
 * the AAS/AAQ column maps (matvct.f:152-170,255-306), MV0303 'X=AY' or
 * 'X=TAY' fills W1..W3 and the diagonal part (mv0303.f:117-165,405-456),
 * ASSVEC adds W into MESH%T (matvct.f:550-560), and MATVEC combines T into
 * X with OS (matvec.f:316-380).  t[npoin] and w[3*nelem] are work arrays
 * (MESH%T and MESH%W). */
int orc_matvec(const char *op, int npoin, int nelem,
               const int *ik0, const int *ik1, const int *ik2,
               double *x, const double *da, char typdia,
               const double *xm, int ld, char typext,
               const double *y, double c, double *t, double *w)
{
    int trans = (strstr(op, "TAY") != NULL);
    const double *xa12, *xa13, *xa23, *xa21, *xa31, *xa32;
    if (typext == 'S') {
        xa12 = xm; xa13 = xm + ld; xa23 = xm + 2 * (size_t)ld;
        xa21 = xa12; xa31 = xa13; xa32 = xa23;
    } else if (typext == 'Q') {
        xa12 = xm; xa13 = xm + ld; xa23 = xm + 2 * (size_t)ld;
        xa21 = xm + 3 * (size_t)ld; xa31 = xm + 4 * (size_t)ld;
        xa32 = xm + 5 * (size_t)ld;
    } else if (typext == '0') {
        xa12 = xa13 = xa23 = xa21 = xa31 = xa32 = NULL;
    } else {
        return ORC_ERR_ARGS;
    }
    double *w1 = w, *w2 = w + nelem, *w3 = w + 2 * (size_t)nelem;
    if (xa12 == NULL) {
        for (int e = 0; e < nelem; ++e) w1[e] = w2[e] = w3[e] = 0.0;
    } else if (!trans) {
        for (int e = 0; e < nelem; ++e) {
            w1[e] = xa12[e] * y[ik1[e]] + xa13[e] * y[ik2[e]];
            w2[e] = xa23[e] * y[ik2[e]] + xa21[e] * y[ik0[e]];
            w3[e] = xa31[e] * y[ik0[e]] + xa32[e] * y[ik1[e]];
        }
    } else {
        for (int e = 0; e < nelem; ++e) {
            w1[e] = xa21[e] * y[ik1[e]] + xa31[e] * y[ik2[e]];
            w2[e] = xa12[e] * y[ik0[e]] + xa32[e] * y[ik2[e]];
            w3[e] = xa13[e] * y[ik0[e]] + xa23[e] * y[ik1[e]];
        }
    }
    if (typdia == 'Q') {
        for (int i = 0; i < npoin; ++i) t[i] = y[i] * da[i];
    } else if (typdia == 'I') {
        for (int i = 0; i < npoin; ++i) t[i] = y[i];
    } else if (typdia == '0') {
        for (int i = 0; i < npoin; ++i) t[i] = 0.0;
    } else {
        return ORC_ERR_ARGS;
    }
    orc_assvec(t, npoin, nelem, ik0, ik1, ik2, w1, w2, w3, 0);

    const char *tail = op + 2; /* matvec.f compares OP(3:8) */
    if (!trans) {
        if (!strncmp(tail, "AY", 2) && (tail[2] == ' ' || tail[2] == 0)) {
            for (int i = 0; i < npoin; ++i) x[i] = t[i];
        } else if (!strncmp(tail, "X+AY", 4)) {
            for (int i = 0; i < npoin; ++i) x[i] = x[i] + t[i];
        } else if (!strncmp(tail, "-AY", 3)) {
            for (int i = 0; i < npoin; ++i) x[i] = -t[i];
        } else if (!strncmp(tail, "X-AY", 4)) {
            for (int i = 0; i < npoin; ++i) x[i] = x[i] - t[i];
        } else if (!strncmp(tail, "X+CAY", 5)) {
            for (int i = 0; i < npoin; ++i) x[i] = x[i] + c * t[i];
        } else if (!strncmp(tail, "CAY", 3)) {
            for (int i = 0; i < npoin; ++i) x[i] = c * t[i];
        } else {
            return ORC_ERR_ARGS;
        }
    } else {
        if (!strncmp(tail, "TAY", 3)) {
            for (int i = 0; i < npoin; ++i) x[i] = t[i];
        } else if (!strncmp(tail, "-TAY", 4)) {
            for (int i = 0; i < npoin; ++i) x[i] = -t[i];
        } else if (!strncmp(tail, "X+TAY", 5)) {
            for (int i = 0; i < npoin; ++i) x[i] = x[i] + t[i];
        } else if (!strncmp(tail, "X-TAY", 5)) {
            for (int i = 0; i < npoin; ++i) x[i] = x[i] - t[i];
        } else if (!strncmp(tail, "X+CTAY", 6)) {
            for (int i = 0; i < npoin; ++i) x[i] = x[i] + c * t[i];
        } else {
            return ORC_ERR_ARGS;
        }
    }
    return ORC_OK;
}

/* mvseg.f:110-720 -- MATVEC on segment storage (STO=3, P1): X takes the
 * diagonal contribution through OV (ov.f:177-324 formulas), then for
 * ISEG = 1..NSEG, in that order,
 *   X(GLOSEG1) = X(GLOSEG1) +/- [C*]XA1(ISEG)*Y(GLOSEG2)
 *   X(GLOSEG2) = X(GLOSEG2) +/- [C*]XA2(ISEG)*Y(GLOSEG1)
 * with XA1/XA2 swapped for the transposed operations.  xa holds XA(NSEG)
 * for TYPEXT 'S' (XA1 = XA2) or XA(NSEG,2) for 'Q' (matvct.f:681-688).
 * g1/g2 are the 0-based GLOSEG columns. */
int orc_mvseg(const char *op, int npoin, int nseg, const int *g1, const int *g2,
              double *x, const double *da, char typdia, const double *xa,
              char typext, const double *y, double c)
{
    char o[9];
    int n = 0;
    for (; n < 8 && op[n]; ++n) o[n] = op[n];
    while (n > 0 && o[n - 1] == ' ') --n;
    o[n] = 0;
    /* dk: diagonal form (0 X=D, 1 X=cD, 2 X=-D, 3 X=X+D, 4 X=X-D, 5 X=X+cD);
     * neg: subtract the segment terms; cm: multiply XA by C; tr: transposed */
    int dk, neg = 0, cm = 0, tr = 0;
    if (!strcmp(o, "X=AY")) dk = 0;
    else if (!strcmp(o, "X=CAY")) { dk = 1; cm = 1; }
    else if (!strcmp(o, "X=-AY")) { dk = 2; neg = 1; }
    else if (!strcmp(o, "X=X+AY")) dk = 3;
    else if (!strcmp(o, "X=X-AY")) { dk = 4; neg = 1; }
    else if (!strcmp(o, "X=X+CAY")) { dk = 5; cm = 1; }
    else if (!strcmp(o, "X=TAY")) { dk = 0; tr = 1; }
    else if (!strcmp(o, "X=-TAY")) { dk = 2; neg = 1; tr = 1; }
    else if (!strcmp(o, "X=X+TAY")) { dk = 3; tr = 1; }
    else if (!strcmp(o, "X=X-TAY")) { dk = 4; neg = 1; tr = 1; }
    else if (!strcmp(o, "X=X+CTAY")) { dk = 5; cm = 1; tr = 1; }
    else return ORC_ERR_ARGS;
    if (typdia != 'Q' && typdia != 'I' && typdia != '0') return ORC_ERR_ARGS;
    for (int i = 0; i < npoin; ++i) {
        double d = typdia == 'Q' ? y[i] * da[i] : y[i];        /* OV 'X=YZ' / 'X=Y' */
        double cd = typdia == 'Q' ? c * y[i] * da[i] : c * y[i]; /* 'X=CYZ' / 'X=CY' */
        if (typdia == '0') {
            if (dk <= 2) x[i] = 0.0;                            /* OV 'X=C' with 0 */
            continue;                                           /* X+.. : no term */
        }
        switch (dk) {
            case 0: x[i] = d; break;
            case 1: x[i] = cd; break;
            case 2: x[i] = -d; break;
            case 3: x[i] = x[i] + d; break;
            case 4: x[i] = x[i] - d; break;
            default: x[i] = x[i] + cd; break;
        }
    }
    if (typext == '0') return ORC_OK;
    if (typext != 'S' && typext != 'Q') return ORC_ERR_ARGS;
    const double *xa1 = xa, *xa2 = typext == 'Q' ? xa + nseg : xa;
    if (tr) { const double *t = xa1; xa1 = xa2; xa2 = t; }
    for (int s = 0; s < nseg; ++s) {
        double a1 = cm ? c * xa1[s] : xa1[s], a2 = cm ? c * xa2[s] : xa2[s];
        if (neg) {
            x[g1[s]] = x[g1[s]] - a1 * y[g2[s]];
            x[g2[s]] = x[g2[s]] - a2 * y[g1[s]];
        } else {
            x[g1[s]] = x[g1[s]] + a1 * y[g2[s]];
            x[g2[s]] = x[g2[s]] + a2 * y[g1[s]];
        }
    }
    return ORC_OK;
}

/* The operator of a solve: EBE (STO=1) or segment (STO=3) storage. */
typedef struct {
    int sto;
    int nelem, ld;
    const int *ik0, *ik1, *ik2;
    int nseg;
    const int *g1, *g2;
    /* node -> (element, local point) index in ASSVEC order, set only when
     * the solve runs on several threads (op_matvec's gather form) */
    const int *gptr, *gek;
} opmesh;

/* MATVEC 'X=AY' for symmetric EBE storage as a per-node gather: node i
 * starts from MATVCT's diagonal term and adds, in ASSVEC's order (local
 * point, then element), the W(e,k) that MV0303 forms for it -- the
 * additions orc_matvec's scatter makes into T(i), in the same order, so the
 * same bits, but every node independent of the others. */
static void mv_ay_gather(const opmesh *M, int npoin, double *x, const double *da,
                         char typdia, const double *xm, const double *y)
{
    const int *ik[3] = {M->ik0, M->ik1, M->ik2};
    const double *xa12 = xm, *xa13 = xm + M->ld, *xa23 = xm + 2 * (size_t)M->ld;
    const int *ptr = M->gptr, *ek = M->gek;
    #pragma omp parallel for if (ORC_PAR(npoin)) num_threads(orc_nthreads) schedule(static)
    for (int i = 0; i < npoin; ++i) {
        double t = typdia == 'Q' ? y[i] * da[i] : (typdia == 'I' ? y[i] : 0.0);
        for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
            int e = ek[j] >> 2, k = ek[j] & 3;
            double w;
            if (k == 0)      w = xa12[e] * y[ik[1][e]] + xa13[e] * y[ik[2][e]];
            else if (k == 1) w = xa23[e] * y[ik[2][e]] + xa12[e] * y[ik[0][e]];
            else             w = xa13[e] * y[ik[0][e]] + xa23[e] * y[ik[1][e]];
            t = t + w;
        }
        x[i] = t;
    }
}

static int op_matvec(const opmesh *M, const char *op, int npoin, double *x,
                     const double *da, char typdia, const double *xm,
                     char typext, const double *y, double c, double *t, double *w)
{
    if (M->sto == 3)
        return orc_mvseg(op, npoin, M->nseg, M->g1, M->g2, x, da, typdia, xm, typext, y, c);
    if (M->gptr && typext == 'S' && !strcmp(op, "X=AY    ") &&
        (typdia == 'Q' || typdia == 'I' || typdia == '0')) {
        mv_ay_gather(M, npoin, x, da, typdia, xm, y);
        return ORC_OK;
    }
    return orc_matvec(op, npoin, M->nelem, M->ik0, M->ik1, M->ik2, x, da, typdia, xm,
                      M->ld, typext, y, c, t, w);
}

static int build_gather(int npoin, int nelem, const int *ik0, const int *ik1,
                        const int *ik2, int **ptr_out, int **ek_out);

/* ------------------------------------------------------------------ */
/* dot products                                                         */
/* ------------------------------------------------------------------ */

/* dot.f:50-54 -- sequential left-to-right sum (P_DOTS with NCSIZE<=1,
 * p_dots.f:146-149). */
double orc_dot(int n, const double *x, const double *y)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = s + x[i] * y[i];
    return s;
}

/* The device kernels' fixed summation tree for a block of `nt` thread
 * partials: a xor-butterfly inside each 32-lane warp (offsets 16..1),
 * then the warp totals (zero-padded to 32) through one more butterfly. */
static double tree64(const double *v, int nt)
{
    double lanes[32], wsum[32];
    int nw = nt / 32;
    for (int w = 0; w < 32; ++w) wsum[w] = 0.0;
    for (int w = 0; w < nw; ++w) {
        for (int l = 0; l < 32; ++l) lanes[l] = v[w * 32 + l];
        for (int o = 16; o >= 1; o >>= 1) {
            double nxt[32];
            for (int l = 0; l < 32; ++l) nxt[l] = lanes[l] + lanes[l ^ o];
            memcpy(lanes, nxt, sizeof(lanes));
        }
        wsum[w] = lanes[0];
    }
    for (int o = 16; o >= 1; o >>= 1) {
        double nxt[32];
        for (int l = 0; l < 32; ++l) nxt[l] = wsum[l] + wsum[l ^ o];
        memcpy(wsum, nxt, sizeof(wsum));
    }
    return wsum[0];
}

static float tree32(const float *v, int nt)
{
    float lanes[32], wsum[32];
    int nw = nt / 32;
    for (int w = 0; w < 32; ++w) wsum[w] = 0.0f;
    for (int w = 0; w < nw; ++w) {
        for (int l = 0; l < 32; ++l) lanes[l] = v[w * 32 + l];
        for (int o = 16; o >= 1; o >>= 1) {
            float nxt[32];
            for (int l = 0; l < 32; ++l) nxt[l] = lanes[l] + lanes[l ^ o];
            memcpy(lanes, nxt, sizeof(lanes));
        }
        wsum[w] = lanes[0];
    }
    for (int o = 16; o >= 1; o >>= 1) {
        float nxt[32];
        for (int l = 0; l < 32; ++l) nxt[l] = wsum[l] + wsum[l ^ o];
        memcpy(wsum, nxt, sizeof(wsum));
    }
    return wsum[0];
}

/* Node range of block b: [blk_lo(b), blk_lo(b+1)), starts rounded down to
 * a multiple of 32 so that every warp's nodes lie in one 32-node slice. */
static long long blk_lo(int b, int n, int nb)
{
    if (b >= nb) return n;
    return ((long long)b * n / nb) & ~31LL;
}

/* The device kernels' dot order: block b owns nodes
 * [b*n/nb, (b+1)*n/nb); thread t sums nodes lo+t, lo+t+nt, ... left to
 * right; the block's nt partials go through tree64; the nb block partials
 * are summed the same way (thread t: partials t, t+nt, ...; then tree64). */
double orc_dot_blocked(int n, const double *x, const double *y,
                       int nb, int nt)
{
    if (nt < 32 || nt > ORC_MAX_NT) return NAN;
    double *part = (double *)malloc(sizeof(double) * (size_t)nb);
    double v[ORC_MAX_NT];
    #pragma omp parallel for if (ORC_PAR(n)) num_threads(orc_nthreads) schedule(static)
    for (int b = 0; b < nb; ++b) {
        double vb[ORC_MAX_NT];
        long long lo = blk_lo(b, n, nb), hi = blk_lo(b + 1, n, nb);
        for (int t = 0; t < nt; ++t) {
            double s = 0.0;
            for (long long i = lo + t; i < hi; i += nt) s = s + x[i] * y[i];
            vb[t] = s;
        }
        part[b] = tree64(vb, nt);
    }
    for (int t = 0; t < nt; ++t) {
        double s = 0.0;
        for (int b = t; b < nb; b += nt) s = s + part[b];
        v[t] = s;
    }
    double r = tree64(v, nt);
    free(part);
    return r;
}

static float dot_blocked32(int n, const float *x, const float *y, int nb, int nt)
{
    if (nt < 32 || nt > ORC_MAX_NT) return NAN;
    float *part = (float *)malloc(sizeof(float) * (size_t)nb);
    float v[ORC_MAX_NT];
    #pragma omp parallel for if (ORC_PAR(n)) num_threads(orc_nthreads) schedule(static)
    for (int b = 0; b < nb; ++b) {
        float vb[ORC_MAX_NT];
        long long lo = blk_lo(b, n, nb), hi = blk_lo(b + 1, n, nb);
        for (int t = 0; t < nt; ++t) {
            float s = 0.0f;
            for (long long i = lo + t; i < hi; i += nt) s = s + x[i] * y[i];
            vb[t] = s;
        }
        part[b] = tree32(vb, nt);
    }
    for (int t = 0; t < nt; ++t) {
        float s = 0.0f;
        for (int b = t; b < nb; b += nt) s = s + part[b];
        v[t] = s;
    }
    float r = tree32(v, nt);
    free(part);
    return r;
}

/* The batched solver's dot order for one instance of n nodes: tiles of
 * C = nt*npt consecutive nodes; in a tile, thread t sums nodes t, t+nt, ...
 * (npt of them) left to right and the nt thread sums go through tree64;
 * the instance total is a 32-lane warp sum: lane l adds tile partials l,
 * l+32, ... left to right, then a xor-butterfly (offsets 16..1). */
static double warp_tree64(double *lanes)
{
    for (int o = 16; o >= 1; o >>= 1) {
        double nxt[32];
        for (int l = 0; l < 32; ++l) nxt[l] = lanes[l] + lanes[l ^ o];
        memcpy(lanes, nxt, sizeof(nxt));
    }
    return lanes[0];
}

static float warp_tree32(float *lanes)
{
    for (int o = 16; o >= 1; o >>= 1) {
        float nxt[32];
        for (int l = 0; l < 32; ++l) nxt[l] = lanes[l] + lanes[l ^ o];
        memcpy(lanes, nxt, sizeof(nxt));
    }
    return lanes[0];
}

double orc_dot_batch(int n, const double *x, const double *y, int nt, int npt)
{
    const int C = nt * npt, ntile = (n + C - 1) / C;
    if (nt < 32 || nt > ORC_MAX_NT) return NAN;
    double *part = (double *)malloc(sizeof(double) * (size_t)(ntile + 1));
    #pragma omp parallel for if (ORC_PAR(n)) num_threads(orc_nthreads) schedule(static)
    for (int k = 0; k < ntile; ++k) {
        double v[ORC_MAX_NT];
        for (int t = 0; t < nt; ++t) {
            double s = 0.0;
            for (int j = 0; j < npt; ++j) {
                long long i = (long long)k * C + t + (long long)j * nt;
                if (i < n) s = s + x[i] * y[i];
            }
            v[t] = s;
        }
        part[k] = tree64(v, nt);
    }
    double lanes[32];
    for (int l = 0; l < 32; ++l) {
        double s = 0.0;
        for (int k = l; k < ntile; k += 32) s = s + part[k];
        lanes[l] = s;
    }
    double r = warp_tree64(lanes);
    free(part);
    return r;
}

static float dot_batch32(int n, const float *x, const float *y, int nt, int npt)
{
    const int C = nt * npt, ntile = (n + C - 1) / C;
    if (nt < 32 || nt > ORC_MAX_NT) return NAN;
    float *part = (float *)malloc(sizeof(float) * (size_t)(ntile + 1));
    #pragma omp parallel for if (ORC_PAR(n)) num_threads(orc_nthreads) schedule(static)
    for (int k = 0; k < ntile; ++k) {
        float v[ORC_MAX_NT];
        for (int t = 0; t < nt; ++t) {
            float s = 0.0f;
            for (int j = 0; j < npt; ++j) {
                long long i = (long long)k * C + t + (long long)j * nt;
                if (i < n) s = s + x[i] * y[i];
            }
            v[t] = s;
        }
        part[k] = tree32(v, nt);
    }
    float lanes[32];
    for (int l = 0; l < 32; ++l) {
        float s = 0.0f;
        for (int k = l; k < ntile; k += 32) s = s + part[k];
        lanes[l] = s;
    }
    float r = warp_tree32(lanes);
    free(part);
    return r;
}

/* ------------------------------------------------------------------ */
/* compensated dot products (MODASS = 3)                                */
/* ------------------------------------------------------------------ */

/* twosum.f: X = A+B, Y = (A-(X-Z))+(B-Z) with Z = X-A (the exact error). */
static void two_sum(double a, double b, double *x, double *y)
{
    double xo = a + b, z = xo - a;
    *y = (a - (xo - z)) + (b - z);
    *x = xo;
}

/* twoprod.f with split.f (Dekker, constant 2**27+1): X = A*B and the exact
 * error Y of that product. */
static void split27(double a, double *x, double *y)
{
    double z = 134217729.0 * a;
    *x = z - (z - a);
    *y = a - *x;
}

static void two_prod(double a, double b, double *x, double *y)
{
    double ah, al, bh, bl;
    *x = a * b;
    split27(a, &ah, &al);
    split27(b, &bh, &bl);
    *y = al * bl - (((*x - ah * bh) - al * bh) - ah * bl);
}

/* dot_comp.f:50-70 -- Dot2 in the reference's sequential order. */
double orc_dot_comp(int n, const double *x, const double *y)
{
    if (n == 0) return 0.0;
    double p, s, h, r, q;
    two_prod(x[0], y[0], &p, &s);
    for (int i = 1; i < n; ++i) {
        two_prod(x[i], y[i], &h, &r);
        two_sum(p, h, &p, &q);
        s = s + (q + r);
    }
    return p + s;
}

/* The device's compensated dot (blocked order): each thread runs Dot2 over
 * its nodes from (p, s) = (0, 0); pairs merge as (p, q) = TwoSum(p1, p2),
 * s = (s1 + s2) + q, through the same xor-butterfly trees as the plain
 * blocked dot; the result is p + s. */
typedef struct { double p, s; } cpair;

static cpair cmerge(cpair a, cpair b)
{
    cpair r;
    double q;
    two_sum(a.p, b.p, &r.p, &q);
    r.s = (a.s + b.s) + q;
    return r;
}

static cpair ctree(const cpair *v, int nt)
{
    cpair lanes[32], wsum[32], nxt[32];
    int nw = nt / 32;
    for (int w = 0; w < 32; ++w) { wsum[w].p = 0.0; wsum[w].s = 0.0; }
    for (int w = 0; w < nw; ++w) {
        for (int l = 0; l < 32; ++l) lanes[l] = v[w * 32 + l];
        for (int o = 16; o >= 1; o >>= 1) {
            for (int l = 0; l < 32; ++l) nxt[l] = cmerge(lanes[l], lanes[l ^ o]);
            memcpy(lanes, nxt, sizeof(lanes));
        }
        wsum[w] = lanes[0];
    }
    for (int o = 16; o >= 1; o >>= 1) {
        for (int l = 0; l < 32; ++l) nxt[l] = cmerge(wsum[l], wsum[l ^ o]);
        memcpy(wsum, nxt, sizeof(wsum));
    }
    return wsum[0];
}

double orc_dot_blocked_comp(int n, const double *x, const double *y, int nb, int nt)
{
    cpair *part = (cpair *)malloc(sizeof(cpair) * (size_t)nb);
    cpair *v = (cpair *)malloc(sizeof(cpair) * (size_t)nt);
    for (int b = 0; b < nb; ++b) {
        long long lo = blk_lo(b, n, nb), hi = blk_lo(b + 1, n, nb);
        for (int t = 0; t < nt; ++t) {
            cpair a = {0.0, 0.0};
            for (long long i = lo + t; i < hi; i += nt) {
                double h, r, q;
                two_prod(x[i], y[i], &h, &r);
                two_sum(a.p, h, &a.p, &q);
                a.s = a.s + (q + r);
            }
            v[t] = a;
        }
        part[b] = ctree(v, nt);
    }
    for (int t = 0; t < nt; ++t) {
        cpair a = {0.0, 0.0};
        for (int b = t; b < nb; b += nt) a = cmerge(a, part[b]);
        v[t] = a;
    }
    cpair r = ctree(v, nt);
    free(part); free(v);
    return r.p + r.s;
}

/* Dot-product order used by the mixed-precision solvers: the persistent
 * single-mesh kernel's blocked order (nb blocks of nt threads) or the
 * batched kernel's tiled order (nt threads, npt nodes per thread). */
typedef struct { int batch; int nb; int nt; int npt; } dotspec;

static double dot64s(const dotspec *ds, int n, const double *x, const double *y)
{
    return ds->batch ? orc_dot_batch(n, x, y, ds->nt, ds->npt)
                     : orc_dot_blocked(n, x, y, ds->nb, ds->nt);
}

static float dot32s(const dotspec *ds, int n, const float *x, const float *y)
{
    return ds->batch ? dot_batch32(n, x, y, ds->nt, ds->npt)
                     : dot_blocked32(n, x, y, ds->nb, ds->nt);
}

static double pdots(int mode, int n, const double *x, const double *y,
                    int nb, int nt)
{
    switch (mode) {
        case ORC_DOT_BLOCKED: return orc_dot_blocked(n, x, y, nb, nt);
        case ORC_DOT_COMP_SEQUENTIAL: return orc_dot_comp(n, x, y);
        case ORC_DOT_COMP_BLOCKED: return orc_dot_blocked_comp(n, x, y, nb, nt);
        default: return orc_dot(n, x, y);
    }
}

/* ------------------------------------------------------------------ */
/* diagonal preconditioning                                             */
/* ------------------------------------------------------------------ */

/* precd1.f:88-158 with DIADON=.FALSE., PREXSM=.TRUE., NCSIZE<=1:
 *   D = A%D; [PRECON=5: D=|D|]; D = SQRT(D); X = X*D;
 *   D = 1/D guarded (ovd.f:92-102, IOPT=2: |D|>1e-10 ? 1/D : 1.0);
 *   A = D*A*D (om.f:249-255 -> om1111.f:559-600);
 *   PRECON divisible by 2 or 3: TYPDIA = 'I' (precd1.f:137-142);
 *   B = B*D.
 * d[npoin] receives D (the reference's TBB(IT1)). */
static int precd1_impl(const opmesh *M, int npoin, int precon, double *x, double *dm,
                       char *typdia, double *xm, char typext, double *b, double *d)
{
    const int nelem = M->nelem, ld = M->ld;
    const int *ik0 = M->ik0, *ik1 = M->ik1, *ik2 = M->ik2;
    for (int i = 0; i < npoin; ++i) d[i] = dm[i];
    if (precon == 5)
        for (int i = 0; i < npoin; ++i) d[i] = fabs(d[i]);
    for (int i = 0; i < npoin; ++i) d[i] = sqrt(d[i]);
    for (int i = 0; i < npoin; ++i) x[i] = x[i] * d[i];
    for (int i = 0; i < npoin; ++i)
        d[i] = (fabs(d[i]) > 1.0e-10) ? 1.0 / d[i] : 1.0;
    /* OM1111 'M=DMD': diagonal part */
    if (*typdia == 'Q') {
        for (int i = 0; i < npoin; ++i) dm[i] = dm[i] * d[i];
        for (int i = 0; i < npoin; ++i) dm[i] = dm[i] * d[i];
    } else if (*typdia == 'I') {
        for (int i = 0; i < npoin; ++i) dm[i] = d[i] * d[i];
        *typdia = 'Q';
    } else if (*typdia != '0') {
        return ORC_ERR_ARGS;
    }
    if (M->sto == 3) {
        /* OMSEG 'M=DMD': off-diagonal part (omseg.f:530-541) */
        if (typext == 'S' || typext == 'Q') {
            for (int s = 0; s < M->nseg; ++s)
                xm[s] = xm[s] * d[M->g1[s]] * d[M->g2[s]];
            if (typext == 'Q')
                for (int s = 0; s < M->nseg; ++s)
                    xm[M->nseg + s] = xm[M->nseg + s] * d[M->g1[s]] * d[M->g2[s]];
        }
    } else if (typext == 'S' || typext == 'Q') {
        /* OM1111 'M=DMD': off-diagonal part (om1111.f:589-600) */
        double *x1 = xm, *x2 = xm + ld, *x3 = xm + 2 * (size_t)ld;
        #pragma omp parallel for if (ORC_PAR(nelem)) num_threads(orc_nthreads) schedule(static)
        for (int e = 0; e < nelem; ++e) {
            x1[e] = x1[e] * d[ik1[e]] * d[ik0[e]];
            x2[e] = x2[e] * d[ik2[e]] * d[ik0[e]];
            x3[e] = x3[e] * d[ik2[e]] * d[ik1[e]];
        }
        if (typext == 'Q') {
            double *x4 = xm + 3 * (size_t)ld, *x5 = xm + 4 * (size_t)ld,
                   *x6 = xm + 5 * (size_t)ld;
            for (int e = 0; e < nelem; ++e) {
                x4[e] = x4[e] * d[ik1[e]] * d[ik0[e]];
                x5[e] = x5[e] * d[ik2[e]] * d[ik0[e]];
                x6[e] = x6[e] * d[ik2[e]] * d[ik1[e]];
            }
        }
    }
    if (precon % 2 == 0 || precon % 3 == 0) *typdia = 'I';
    for (int i = 0; i < npoin; ++i) b[i] = b[i] * d[i];
    return ORC_OK;
}

int orc_precd1(int npoin, int nelem, const int *ik0, const int *ik1,
               const int *ik2, int precon, double *x, double *dm,
               char *typdia, double *xm, int ld, char typext, double *b,
               double *d)
{
    opmesh M = {1, nelem, ld, ik0, ik1, ik2, 0, NULL, NULL};
    return precd1_impl(&M, npoin, precon, x, dm, typdia, xm, typext, b, d);
}

/* ------------------------------------------------------------------ */
/* conjugate gradient                                                   */
/* ------------------------------------------------------------------ */

/* gracjg.F:169-437 without preconditioning matrices (PRECON 1/2/3/5 fold
 * into the change of variables done by PRECD1, so G aliases R).
 * Convention R = A X - B; stop when RMRM <= XL*EPS**2 or M = NITMAX.
 * Returns ORC_OK, or the iteration count (>0) when NITMAX was reached
 * without convergence, or a negative error. */
static int gracjg_impl(const opmesh *M, int npoin, double *x, const double *da,
                       char typdia, const double *xm, char typext, const double *b,
                       int nitmax, double eps, int dot_mode, int nb, int nt,
                       int *nit_out, double *relres_out, int *relat_out)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *r = (double *)malloc(sizeof(double) * n);
    double *dd = (double *)malloc(sizeof(double) * n);
    double *ad = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int m = 0, st = ORC_OK, relat;
    double xl, rmrm, rmgm, rmdm, rm1gm1, dad, ro, beta;
    if (!r || !dd || !ad || !t || !w) { st = ORC_ERR_ARGS; goto done; }

    xl = pdots(dot_mode, npoin, b, b, nb, nt);            /* :189 */
    if (sqrt(xl) < 1.0e-15) {                             /* :194-202 */
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) x[i] = 0.0;
        rmrm = 0.0; xl = 1.0; relat = 0;
        goto fin;
    }
    if (xl < 1.0) { xl = 1.0; relat = 0; } else { relat = 1; }  /* :204-209 */

    st = op_matvec(M, "X=AY    ", npoin, r, da, typdia, xm, typext, x, 0.0, t, w);  /* :213 */
    if (st) goto done;
    ORC_PFOR(n)
    for (size_t i = 0; i < n; ++i) r[i] = r[i] - b[i];    /* :215 */
    rmrm = pdots(dot_mode, npoin, r, r, nb, nt);          /* :216 */
    rmgm = rmrm;
    if (rmrm < eps * eps * xl) goto fin;                  /* :219 */

    ORC_PFOR(n)
    for (size_t i = 0; i < n; ++i) dd[i] = r[i];          /* :248 */
    st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t, w); /* :254 */
    if (st) goto done;
    dad = pdots(dot_mode, npoin, dd, ad, nb, nt);         /* :260 */
    ro = rmgm / dad;                                      /* :261 */
    ORC_PFOR(n)
    for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];   /* :268 */

    for (;;) {
        m = m + 1;                                        /* :284 */
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) r[i] = r[i] + (-ro) * ad[i];  /* :290 */
        rm1gm1 = rmgm;
        rmrm = pdots(dot_mode, npoin, r, r, nb, nt);      /* :295 */
        rmdm = rmrm;
        rmgm = rmrm;
        if (rmrm <= xl * (eps * eps)) goto fin;           /* :303,324 */
        beta = rmgm / rm1gm1;                             /* :357 */
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) dd[i] = r[i] + beta * dd[i];  /* :361 */
        st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t,
                       w);                                /* :376 */
        if (st) goto done;
        dad = pdots(dot_mode, npoin, dd, ad, nb, nt);     /* :382 */
        ro = rmdm / dad;                                  /* :383 */
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];  /* :387 */
        if (m >= nitmax) { st = m; goto fin; }            /* :406 */
    }
fin:
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = sqrt(rmrm / xl);
    if (relat_out) *relat_out = relat;
done:
    free(r); free(dd); free(ad); free(t); free(w);
    return st;
}

int orc_gracjg(int npoin, int nelem, const int *ik0, const int *ik1,
               const int *ik2, double *x, const double *da, char typdia,
               const double *xm, int ld, char typext, const double *b,
               int nitmax, double eps, int dot_mode, int nb, int nt,
               int *nit_out, double *relres_out, int *relat_out)
{
    opmesh M = {1, nelem, ld, ik0, ik1, ik2, 0, NULL, NULL};
    return gracjg_impl(&M, npoin, x, da, typdia, xm, typext, b, nitmax, eps, dot_mode, nb, nt,
                       nit_out, relres_out, relat_out);
}

/* equnor.f:106-311 (CG on the normal equations) without preconditioning
 * matrices (PREC false, so G aliases R, solve.f:473-474):
 *   XL = B.B (absolute mode below 1); R = A X - B; RMRM = R.R; stop if
 *   RMRM < EPS**2 XL; D = A^T R; TGMTGM = D.D; AD = A D; RO = TGMTGM/AD.AD;
 *   X = X - RO D; then per iteration R = R - RO AD; RMRM = R.R; stop if
 *   RMRM <= XL EPS**2; AD = A^T R; BETA = AD.AD / previous TGMTGM;
 *   D = BETA D, D = D + AD (two passes, 'X=CX' then 'X=X+Y'); AD = A D;
 *   RO = TGMTGM / AD.AD; X = X - RO D; stop at NITMAX. */
static int equnor_impl(const opmesh *M, int npoin, double *x, const double *da, char typdia,
                       const double *xm, char typext, const double *b, int nitmax, double eps,
                       int dot_mode, int nb, int nt, int *nit_out, double *relres_out,
                       int *relat_out)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *r = (double *)malloc(sizeof(double) * n);
    double *dd = (double *)malloc(sizeof(double) * n);
    double *ad = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int m = 0, st = ORC_OK, relat;
    double xl, rmrm, tgmtgm, tg1tg1, adad, ro, beta;
    if (!r || !dd || !ad || !t || !w) { st = ORC_ERR_ARGS; goto done; }
    xl = pdots(dot_mode, npoin, b, b, nb, nt);                    /* :108 */
    if (xl < 1.0) { xl = 1.0; relat = 0; } else { relat = 1; }    /* :109-114 */
    st = op_matvec(M, "X=AY    ", npoin, r, da, typdia, xm, typext, x, 0.0, t, w);  /* :118 */
    if (st) goto done;
    for (size_t i = 0; i < n; ++i) r[i] = r[i] - b[i];          /* :119 */
    rmrm = pdots(dot_mode, npoin, r, r, nb, nt);                 /* :123 */
    if (rmrm < eps * eps * xl) goto fin;                         /* :127 */
    st = op_matvec(M, "X=TAY   ", npoin, dd, da, typdia, xm, typext, r, 0.0, t, w); /* :160 */
    if (st) goto done;
    tgmtgm = pdots(dot_mode, npoin, dd, dd, nb, nt);             /* :163 */
    st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t, w); /* :169 */
    if (st) goto done;
    adad = pdots(dot_mode, npoin, ad, ad, nb, nt);               /* :187 */
    ro = tgmtgm / adad;                                          /* :189 */
    for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];  /* :195 */
    for (;;) {
        m = m + 1;                                               /* :201 */
        for (size_t i = 0; i < n; ++i) r[i] = r[i] + (-ro) * ad[i];      /* :207 */
        rmrm = pdots(dot_mode, npoin, r, r, nb, nt);             /* :211 */
        if (rmrm <= xl * (eps * eps)) goto fin;                  /* :215 */
        st = op_matvec(M, "X=TAY   ", npoin, ad, da, typdia, xm, typext, r, 0.0, t, w); /* :240 */
        if (st) goto done;
        tg1tg1 = tgmtgm;                                         /* :243 */
        tgmtgm = pdots(dot_mode, npoin, ad, ad, nb, nt);         /* :244 */
        beta = tgmtgm / tg1tg1;                                  /* :245 */
        for (size_t i = 0; i < n; ++i) dd[i] = beta * dd[i];     /* :247 */
        for (size_t i = 0; i < n; ++i) dd[i] = dd[i] + ad[i];    /* :250 */
        st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t, w); /* :256 */
        if (st) goto done;
        adad = pdots(dot_mode, npoin, ad, ad, nb, nt);           /* :272 */
        ro = tgmtgm / adad;                                      /* :274 */
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];      /* :278 */
        if (m >= nitmax) { st = m; goto fin; }                   /* :280 */
    }
fin:
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = sqrt(rmrm / xl);
    if (relat_out) *relat_out = relat;
done:
    free(r); free(dd); free(ad); free(t); free(w);
    return st;
}

/* rescjg.f:134-315 (conjugate residual) without preconditioning matrices
 * (G aliases R):  XL = B.B (absolute below 1); R = A X - B; RMRM = R.R; stop
 * if RMRM < EPS**2 XL; D = R; AD = A D; RO = D.AD / AD.AD; X = X - RO D; per
 * iteration R = R - RO AD; RMRM = R.R; stop if RMRM <= XL EPS**2;
 * AG = A R; BETA = -(AG.AD / AD.AD); D = BETA D + R, AD = BETA AD + AG (each
 * as 'X=CX' then 'X=X+Y'); RO = R.AD / AD.AD; X = X - RO D; NITMAX. */
static int rescjg_impl(const opmesh *M, int npoin, double *x, const double *da, char typdia,
                       const double *xm, char typext, const double *b, int nitmax, double eps,
                       int dot_mode, int nb, int nt, int *nit_out, double *relres_out,
                       int *relat_out)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *r = (double *)malloc(sizeof(double) * n), *dd = (double *)malloc(sizeof(double) * n);
    double *ad = (double *)malloc(sizeof(double) * n), *ag = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int m = 0, st = ORC_OK, relat;
    double xl, rmrm, dad, adad, agad, gad, ro, beta;
    if (!r || !dd || !ad || !ag || !t || !w) { st = ORC_ERR_ARGS; goto done; }
    xl = pdots(dot_mode, npoin, b, b, nb, nt);                          /* :134 */
    if (xl < 1.0) { xl = 1.0; relat = 0; } else { relat = 1; }
    st = op_matvec(M, "X=AY    ", npoin, r, da, typdia, xm, typext, x, 0.0, t, w);   /* :144 */
    if (st) goto done;
    for (size_t i = 0; i < n; ++i) r[i] = r[i] - b[i];                 /* :146 */
    rmrm = pdots(dot_mode, npoin, r, r, nb, nt);
    if (rmrm < eps * eps * xl) goto fin;                                /* :149 */
    memcpy(dd, r, sizeof(double) * n);                                  /* :178 */
    st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t, w); /* :184 */
    if (st) goto done;
    dad = pdots(dot_mode, npoin, dd, ad, nb, nt);                       /* :211 */
    adad = pdots(dot_mode, npoin, ad, ad, nb, nt);                      /* :215 */
    ro = dad / adad;
    for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];        /* :223 */
    for (;;) {
        m = m + 1;                                                      /* :229 */
        for (size_t i = 0; i < n; ++i) r[i] = r[i] + (-ro) * ad[i];    /* :235 */
        rmrm = pdots(dot_mode, npoin, r, r, nb, nt);
        if (rmrm <= xl * (eps * eps)) goto fin;                         /* :243 */
        st = op_matvec(M, "X=AY    ", npoin, ag, da, typdia, xm, typext, r, 0.0, t, w); /* :258 */
        if (st) goto done;
        agad = pdots(dot_mode, npoin, ag, ad, nb, nt);                  /* :267 */
        beta = -agad / adad;                                            /* :269 */
        for (size_t i = 0; i < n; ++i) dd[i] = beta * dd[i];           /* :271-272 */
        for (size_t i = 0; i < n; ++i) dd[i] = dd[i] + r[i];
        for (size_t i = 0; i < n; ++i) ad[i] = beta * ad[i];           /* :278-279 */
        for (size_t i = 0; i < n; ++i) ad[i] = ad[i] + ag[i];
        gad = pdots(dot_mode, npoin, r, ad, nb, nt);                    /* :303 */
        adad = pdots(dot_mode, npoin, ad, ad, nb, nt);                  /* :307 */
        ro = gad / adad;
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];    /* :313 */
        if (m >= nitmax) { st = m; goto fin; }                          /* :315 */
    }
fin:
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = sqrt(rmrm / xl);
    if (relat_out) *relat_out = relat;
done:
    free(r); free(dd); free(ad); free(ag); free(t); free(w);
    return st;
}

/* errmin.f:116-259 (minimum error) without preconditioning matrices (G
 * aliases R): XL; R = A X - B; RMRM = GMGM = R.R; stop if RMRM < EPS**2 XL;
 * D = A^T R; RO = GMGM / D.D; AD = A D; X = X - RO D; per iteration
 * R = R - RO AD; GM1GM1 = GMGM; RMRM = GMGM = R.R; stop if RMRM <= XL EPS**2;
 * AD = A^T R; BETA = GMGM/GM1GM1; D = BETA D + AD ('X=CX', 'X=X+Y');
 * AD = A D; RO = GMGM / D.D; X = X - RO D; NITMAX. */
static int errmin_impl(const opmesh *M, int npoin, double *x, const double *da, char typdia,
                       const double *xm, char typext, const double *b, int nitmax, double eps,
                       int dot_mode, int nb, int nt, int *nit_out, double *relres_out,
                       int *relat_out)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *r = (double *)malloc(sizeof(double) * n), *dd = (double *)malloc(sizeof(double) * n);
    double *ad = (double *)malloc(sizeof(double) * n), *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int m = 0, st = ORC_OK, relat;
    double xl, rmrm, gmgm, gm1gm1, tg, ddd, ro, beta;
    if (!r || !dd || !ad || !t || !w) { st = ORC_ERR_ARGS; goto done; }
    xl = pdots(dot_mode, npoin, b, b, nb, nt);                          /* :116 */
    if (xl < 1.0) { xl = 1.0; relat = 0; } else { relat = 1; }
    st = op_matvec(M, "X=AY    ", npoin, r, da, typdia, xm, typext, x, 0.0, t, w);   /* :126 */
    if (st) goto done;
    for (size_t i = 0; i < n; ++i) r[i] = r[i] - b[i];                 /* :128 */
    rmrm = pdots(dot_mode, npoin, r, r, nb, nt);
    gmgm = rmrm;
    if (rmrm < eps * eps * xl) goto fin;                                /* :132 */
    st = op_matvec(M, "X=TAY   ", npoin, dd, da, typdia, xm, typext, r, 0.0, t, w); /* :161 */
    if (st) goto done;
    tg = pdots(dot_mode, npoin, dd, dd, nb, nt);                        /* :164 */
    st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t, w); /* :170 */
    if (st) goto done;
    ro = gmgm / tg;                                                     /* :176 */
    for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];        /* :182 */
    for (;;) {
        m = m + 1;                                                      /* :188 */
        for (size_t i = 0; i < n; ++i) r[i] = r[i] + (-ro) * ad[i];    /* :194 */
        gm1gm1 = gmgm;
        rmrm = pdots(dot_mode, npoin, r, r, nb, nt);                    /* :199 */
        gmgm = rmrm;
        if (rmrm <= xl * (eps * eps)) goto fin;                         /* :204 */
        st = op_matvec(M, "X=TAY   ", npoin, ad, da, typdia, xm, typext, r, 0.0, t, w); /* :232 */
        if (st) goto done;
        beta = gmgm / gm1gm1;                                           /* :235 */
        for (size_t i = 0; i < n; ++i) dd[i] = beta * dd[i];           /* :237 */
        for (size_t i = 0; i < n; ++i) dd[i] = dd[i] + ad[i];          /* :240 */
        st = op_matvec(M, "X=AY    ", npoin, ad, da, typdia, xm, typext, dd, 0.0, t, w); /* :246 */
        if (st) goto done;
        ddd = pdots(dot_mode, npoin, dd, dd, nb, nt);                   /* :252 */
        ro = gmgm / ddd;
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * dd[i];    /* :257 */
        if (m >= nitmax) { st = m; goto fin; }                          /* :259 */
    }
fin:
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = sqrt(rmrm / xl);
    if (relat_out) *relat_out = relat;
done:
    free(r); free(dd); free(ad); free(t); free(w);
    return st;
}

/* cgsqua.f:151-282 (conjugate gradient squared):  XL = B.B (absolute below
 * 1); G = A X - B; RL = G.G; stop if RL < EPS**2 XL; G0 = P = K = G; per
 * iteration (M from 1): H = A P; RO = K.G0 / H.G0; H = -RO H, H = H + 2 K;
 * X = X - RO H; AHPK = A H; GMG0 = G.G0; G = G - RO AHPK; RL = G.G; stop if
 * RL <= EPS**2 XL, or at NITMAX; GMP1G0 = G.G0; BETA = GMP1G0 / GMG0;
 * H = H - K; P = BETA**2 P, P = P + G, P = P + 2 BETA H; K = G, K = K + BETA H. */
static int cgsqua_impl(const opmesh *M, int npoin, double *x, const double *da, char typdia,
                       const double *xm, char typext, const double *b, int nitmax, double eps,
                       int dot_mode, int nb, int nt, int *nit_out, double *relres_out,
                       int *relat_out)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *g = (double *)malloc(sizeof(double) * n), *g0 = (double *)malloc(sizeof(double) * n);
    double *p = (double *)malloc(sizeof(double) * n), *k = (double *)malloc(sizeof(double) * n);
    double *h = (double *)malloc(sizeof(double) * n), *ahpk = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int m = 0, st = ORC_OK, relat;
    double xl, rl, ro, kg0, hg0, gmg0, gmp1g0, beta;
    if (!g || !g0 || !p || !k || !h || !ahpk || !t || !w) { st = ORC_ERR_ARGS; goto done; }
    xl = pdots(dot_mode, npoin, b, b, nb, nt);                          /* :151 */
    if (xl < 1.0) { xl = 1.0; relat = 0; } else { relat = 1; }
    st = op_matvec(M, "X=AY    ", npoin, g, da, typdia, xm, typext, x, 0.0, t, w);   /* :164 */
    if (st) goto done;
    for (size_t i = 0; i < n; ++i) g[i] = g[i] - b[i];                 /* :166 */
    rl = pdots(dot_mode, npoin, g, g, nb, nt);                          /* :170 */
    if (rl < eps * eps * xl) goto fin;                                  /* :172 */
    memcpy(g0, g, sizeof(double) * n);                                  /* :188-190 */
    memcpy(p, g, sizeof(double) * n);
    memcpy(k, g, sizeof(double) * n);
    m = 1;
    for (;;) {
        st = op_matvec(M, "X=AY    ", npoin, h, da, typdia, xm, typext, p, 0.0, t, w); /* :197 */
        if (st) goto done;
        kg0 = pdots(dot_mode, npoin, k, g0, nb, nt);                    /* :201 */
        hg0 = pdots(dot_mode, npoin, h, g0, nb, nt);
        ro = kg0 / hg0;
        for (size_t i = 0; i < n; ++i) h[i] = (-ro) * h[i];            /* :205 */
        for (size_t i = 0; i < n; ++i) h[i] = h[i] + 2.0 * k[i];       /* :206 */
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + (-ro) * h[i];     /* :211 */
        st = op_matvec(M, "X=AY    ", npoin, ahpk, da, typdia, xm, typext, h, 0.0, t, w); /* :215 */
        if (st) goto done;
        gmg0 = pdots(dot_mode, npoin, g, g0, nb, nt);                   /* :220 */
        for (size_t i = 0; i < n; ++i) g[i] = g[i] + (-ro) * ahpk[i];  /* :224 */
        rl = pdots(dot_mode, npoin, g, g, nb, nt);                      /* :226 */
        if (!(rl > eps * eps * xl)) goto fin;                           /* :227 */
        if (m >= nitmax) { st = m; goto fin; }                          /* :228 */
        m = m + 1;
        gmp1g0 = pdots(dot_mode, npoin, g, g0, nb, nt);                 /* :258 */
        beta = gmp1g0 / gmg0;                                           /* :262 */
        for (size_t i = 0; i < n; ++i) h[i] = h[i] - k[i];             /* :267 */
        for (size_t i = 0; i < n; ++i) p[i] = (beta * beta) * p[i];    /* :272-274 */
        for (size_t i = 0; i < n; ++i) p[i] = p[i] + g[i];
        for (size_t i = 0; i < n; ++i) p[i] = p[i] + (2.0 * beta) * h[i];
        for (size_t i = 0; i < n; ++i) k[i] = g[i] + beta * h[i];      /* :279-280 */
    }
fin:
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = sqrt(rl / xl);
    if (relat_out) *relat_out = relat;
done:
    free(g); free(g0); free(p); free(k); free(h); free(ahpk); free(t); free(w);
    return st;
}

/* cgstab.f:95-200 (BiCGSTAB) without Crout preconditioning:
 *   XL = B.B (absolute below 1); SQRT(XL) < 1e-15: X = 0; V = A X;
 *   R = B - V; RMRM = R.R; stop if RMRM < EPS**2 XL; R = B, R = R - V
 *   (the same values again); P = R; V = 0; Q = 0; ALFA = BETA = OMEG1 = 1;
 *   per iteration: BETA1 = R.P; OMEG2 = OMEG1*BETA1/BETA;
 *   OMEG = OMEG2/ALFA; BETA = BETA1; Q = R + OMEG Q; Q = Q - OMEG2 V;
 *   V = A Q; OMEG1 = BETA1 / P.V; S = R - OMEG1 V; T = A S;
 *   ALFA = T.S / T.T; X = X + OMEG1 Q; X = X + ALFA S; R = S - ALFA T;
 *   RMRM = R.R; stop if RMRM <= XL EPS**2 or M = NITMAX. */
static int cgstab_impl(const opmesh *M, int npoin, double *x, const double *da, char typdia,
                       const double *xm, char typext, const double *b, int nitmax, double eps,
                       int dot_mode, int nb, int nt, int *nit_out, double *relres_out,
                       int *relat_out)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *p = (double *)malloc(sizeof(double) * n), *q = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n), *sv = (double *)malloc(sizeof(double) * n);
    double *tv = (double *)malloc(sizeof(double) * n), *v = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int m = 0, st = ORC_OK, relat;
    double xl, rmrm = 0.0, alfa, alfa1, beta, beta1, omeg, omeg1, omeg2;
    if (!p || !q || !r || !sv || !tv || !v || !t || !w) { st = ORC_ERR_ARGS; goto done; }
    xl = pdots(dot_mode, npoin, b, b, nb, nt);                       /* :105 */
    if (xl < 1.0) { xl = 1.0; relat = 0; } else { relat = 1; }
    if (sqrt(xl) < 1.0e-15) {                                         /* :112-116 */
        rmrm = 0.0;
        for (size_t i = 0; i < n; ++i) x[i] = 0.0;
        goto fin;
    }
    st = op_matvec(M, "X=AY    ", npoin, v, da, typdia, xm, typext, x, 0.0, t, w);  /* :120 */
    if (st) goto done;
    for (size_t i = 0; i < n; ++i) r[i] = b[i] - v[i];               /* :121 */
    rmrm = pdots(dot_mode, npoin, r, r, nb, nt);
    if (rmrm < eps * eps * xl) goto fin;                             /* :123 */
    for (size_t i = 0; i < n; ++i) r[i] = b[i];                      /* :132 */
    for (size_t i = 0; i < n; ++i) r[i] = r[i] - v[i];               /* :142 */
    for (size_t i = 0; i < n; ++i) { p[i] = r[i]; v[i] = 0.0; q[i] = 0.0; }
    alfa = 1.0; beta = 1.0; omeg1 = 1.0;
    for (;;) {
        m = m + 1;                                                   /* :153 */
        beta1 = pdots(dot_mode, npoin, r, p, nb, nt);
        omeg2 = omeg1 * beta1 / beta;
        omeg = omeg2 / alfa;
        beta = beta1;
        for (size_t i = 0; i < n; ++i) q[i] = r[i] + omeg * q[i];    /* :161 */
        for (size_t i = 0; i < n; ++i) q[i] = q[i] + (-omeg2) * v[i];
        st = op_matvec(M, "X=AY    ", npoin, v, da, typdia, xm, typext, q, 0.0, t, w);
        if (st) goto done;
        omeg1 = pdots(dot_mode, npoin, p, v, nb, nt);                /* :173 */
        omeg1 = beta1 / omeg1;
        for (size_t i = 0; i < n; ++i) sv[i] = r[i] + (-omeg1) * v[i];
        st = op_matvec(M, "X=AY    ", npoin, tv, da, typdia, xm, typext, sv, 0.0, t, w);
        if (st) goto done;
        alfa = pdots(dot_mode, npoin, tv, sv, nb, nt);               /* :186 */
        alfa1 = pdots(dot_mode, npoin, tv, tv, nb, nt);
        alfa = alfa / alfa1;
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + omeg1 * q[i];   /* :190 */
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + alfa * sv[i];
        for (size_t i = 0; i < n; ++i) r[i] = sv[i] + (-alfa) * tv[i];
        rmrm = pdots(dot_mode, npoin, r, r, nb, nt);                 /* :193 */
        if (rmrm <= xl * (eps * eps)) goto fin;
        if (m >= nitmax) { st = m; goto fin; }
    }
fin:
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = sqrt(rmrm / xl);
    if (relat_out) *relat_out = relat;
done:
    free(p); free(q); free(r); free(sv); free(tv); free(v); free(t); free(w);
    return st;
}

/* gmres.f:55-213, restarted GMRES(KRYLOV) without preconditioning
 * matrices (PRECO false), KRYLOV <= 20 (H(21,20)):
 *   NB = SQRT(B.B) (absolute mode below 1); R0 = A X - B; NR0 = |R0|;
 *   stop if NR0/NB <= EPS.  Each restart M: V1 = (-1/NR0) R0; for
 *   J = 1..K-1: AV(J) = A V(J), V(J+1) = AV(J), modified Gram-Schmidt
 *   H(I,J) = V(J+1).V(I), V(J+1) = V(J+1) - H(I,J) V(I) for I = 1..J,
 *   H(J+1,J) = |V(J+1)| (below 1e-20: K = J, leave the loop),
 *   V(J+1) = (1/H(J+1,J)) V(J+1); AV(K) = A V(K); H(K+1,K) =
 *   AV(K).AV(K) - sum of H(I,K)**2 with H(I,K) = AV(K).V(I), then
 *   SQRT(MAX(.,0)); Givens rotations on H and E (E(1) = NR0), R below 1e-6
 *   ends the solve before this restart's update; back substitution;
 *   X = X + E(L) V(L), R0 = R0 + E(L) AV(L) for L = 1..K; NR0 = |E(K+1)|;
 *   restart while NR0/NB >= EPS and M < NITMAX.
 * Returns ORC_OK when M < NITMAX at the end, M (> 0) otherwise (the
 * reference's two end messages); relres_out receives NR0/NB. */
static int gmres_impl(const opmesh *M, int npoin, double *x, const double *da, char typdia,
                      const double *xm, char typext, const double *b, int nitmax, double eps,
                      int krylov, int dot_mode, int nb, int nt, int *nit_out,
                      double *relres_out, int *relat_out)
{
    if (krylov < 1 || krylov > 20) return ORC_ERR_ARGS;
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    size_t n = (size_t)npoin;
    double *r0 = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    double *v = (double *)malloc(sizeof(double) * n * (size_t)krylov);
    double *av = (double *)malloc(sizeof(double) * n * (size_t)krylov);
    double h[21][20], c[20], sn[20], e[21];
    int m = 0, st = ORC_OK, relat = 1;
    double nbn, nr0, prec = 0.0;
    if (!r0 || !t || !w || !v || !av) { st = ORC_ERR_ARGS; goto done; }
#define V(j) (v + (size_t)(j) * n)
#define AV(j) (av + (size_t)(j) * n)
    nbn = sqrt(pdots(dot_mode, npoin, b, b, nb, nt));           /* :67-68 */
    if (nbn < 1.0) { nbn = 1.0; relat = 0; }                     /* :70-73 */
    st = op_matvec(M, "X=AY    ", npoin, r0, da, typdia, xm, typext, x, 0.0, t, w); /* :77 */
    if (st) goto done;
    for (size_t i = 0; i < n; ++i) r0[i] = r0[i] - b[i];        /* :82 */
    nr0 = sqrt(pdots(dot_mode, npoin, r0, r0, nb, nt));          /* :83-84 */
    prec = nr0 / nbn;
    if (prec <= eps) goto fin;                                   /* :87 */
    for (;;) {
        m = m + 1;                                               /* :91 */
        int k = krylov;
        double cc = -1.0 / nr0;
        for (size_t i = 0; i < n; ++i) V(0)[i] = cc * r0[i];     /* :95 */
        for (int j = 1; j <= k - 1; ++j) {                       /* :97-143 */
            st = op_matvec(M, "X=AY    ", npoin, AV(j - 1), da, typdia, xm, typext, V(j - 1),
                           0.0, t, w);
            if (st) goto done;
            memcpy(V(j), AV(j - 1), sizeof(double) * n);
            for (int i = 1; i <= j; ++i) {
                h[i - 1][j - 1] = pdots(dot_mode, npoin, V(j), V(i - 1), nb, nt);
                double ch = -h[i - 1][j - 1];
                for (size_t q = 0; q < n; ++q) V(j)[q] = V(j)[q] + ch * V(i - 1)[q];
            }
            h[j][j - 1] = sqrt(pdots(dot_mode, npoin, V(j), V(j), nb, nt));
            if (h[j][j - 1] < 1.0e-20) { k = j; break; }
            double ci = 1.0 / h[j][j - 1];
            for (size_t q = 0; q < n; ++q) V(j)[q] = ci * V(j)[q];
        }
        st = op_matvec(M, "X=AY    ", npoin, AV(k - 1), da, typdia, xm, typext, V(k - 1), 0.0,
                       t, w);                                    /* :151 */
        if (st) goto done;
        h[k][k - 1] = pdots(dot_mode, npoin, AV(k - 1), AV(k - 1), nb, nt);     /* :153 */
        for (int i = 1; i <= k; ++i) {
            h[i - 1][k - 1] = pdots(dot_mode, npoin, AV(k - 1), V(i - 1), nb, nt);
            h[k][k - 1] = h[k][k - 1] - h[i - 1][k - 1] * h[i - 1][k - 1];
        }
        h[k][k - 1] = sqrt(h[k][k - 1] > 0.0 ? h[k][k - 1] : 0.0);              /* :158 */
        e[0] = nr0;
        for (int i = 1; i <= k; ++i) {                           /* :160-183 */
            for (int j = 1; j <= i - 1; ++j) {
                double zz = c[j - 1] * h[j - 1][i - 1] + sn[j - 1] * h[j][i - 1];
                h[j][i - 1] = -sn[j - 1] * h[j - 1][i - 1] + c[j - 1] * h[j][i - 1];
                h[j - 1][i - 1] = zz;
            }
            double rr = sqrt(h[i - 1][i - 1] * h[i - 1][i - 1] + h[i][i - 1] * h[i][i - 1]);
            if (fabs(rr) < 1.0e-6) goto fin;
            c[i - 1] = h[i - 1][i - 1] / rr;
            sn[i - 1] = h[i][i - 1] / rr;
            h[i - 1][i - 1] = rr;
            e[i] = -sn[i - 1] * e[i - 1];
            e[i - 1] = c[i - 1] * e[i - 1];
        }
        e[k - 1] = e[k - 1] / h[k - 1][k - 1];                   /* :184-190 */
        for (int j = k - 1; j >= 1; --j) {
            for (int l = j + 1; l <= k; ++l) e[j - 1] = e[j - 1] - h[j - 1][l - 1] * e[l - 1];
            e[j - 1] = e[j - 1] / h[j - 1][j - 1];
        }
        for (int l = 1; l <= k; ++l) {                           /* :191-194 */
            for (size_t q = 0; q < n; ++q) x[q] = x[q] + e[l - 1] * V(l - 1)[q];
            for (size_t q = 0; q < n; ++q) r0[q] = r0[q] + e[l - 1] * AV(l - 1)[q];
        }
        nr0 = fabs(e[k]);                                        /* :195 */
        prec = nr0 / nbn;
        if (!(prec >= eps && m < nitmax)) break;                 /* :197 */
    }
#undef V
#undef AV
fin:
    /* the reference reports success whenever M < NITMAX (:199-214), also
     * after the R < 1e-6 failure message; at M = NITMAX it reports the
     * iteration limit */
    st = m < nitmax ? ORC_OK : m;
    if (nit_out) *nit_out = m;
    if (relres_out) *relres_out = prec;
    if (relat_out) *relat_out = relat;
done:
    free(r0); free(t); free(w); free(v); free(av);
    return st;
}

/* solve.f:387-649 for SLV=1 (GRACJG, solve.f:555-558) and SLV=3 (EQUNOR,
 * :565-570) on a single (non-block) matrix:
 * PRECON 0 -> 1; diagonal change of variables when PRECON is divisible by
 * 2, 3 or 5 (solve.f:484-498); CG; X = X*D to undo the change of variables
 * (solve.f:637-641).  Inputs x, b, dm, typdia, xm are modified in place
 * exactly as the reference modifies them. */
static int solve_impl(const opmesh *M, int npoin, double *x, double *b, double *dm,
                      char *typdia, double *xm, char typext, int slv, int precon,
                      int nitmax, double eps, int krylov, int dot_mode, int nb, int nt,
                      int *nit_out, double *relres_out, int *relat_out)
{
    if (slv < 1 || slv > 7) return ORC_ERR_UNSUPPORTED;
    if (precon == 0) precon = 1;
    if (precon % 7 == 0 || precon % 11 == 0 || precon % 13 == 0 ||
        precon % 17 == 0)
        return ORC_ERR_UNSUPPORTED;
    int diag = (precon % 2 == 0 || precon % 3 == 0 || precon % 5 == 0);
    double *d = NULL;
    if (diag) {
        d = (double *)malloc(sizeof(double) * (size_t)npoin);
        int st = precd1_impl(M, npoin, precon, x, dm, typdia, xm, typext, b, d);
        if (st) { free(d); return st; }
    }
    int st = slv == 7
                 ? gmres_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, krylov,
                              dot_mode, nb, nt, nit_out, relres_out, relat_out)
             : slv == 2
                 ? rescjg_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, dot_mode,
                               nb, nt, nit_out, relres_out, relat_out)
             : slv == 4
                 ? errmin_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, dot_mode,
                               nb, nt, nit_out, relres_out, relat_out)
             : slv == 5
                 ? cgsqua_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, dot_mode,
                               nb, nt, nit_out, relres_out, relat_out)
             : slv == 6
                 ? cgstab_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, dot_mode,
                               nb, nt, nit_out, relres_out, relat_out)
             : slv == 3
                 ? equnor_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, dot_mode,
                               nb, nt, nit_out, relres_out, relat_out)
                 : gracjg_impl(M, npoin, x, dm, *typdia, xm, typext, b, nitmax, eps, dot_mode,
                               nb, nt, nit_out, relres_out, relat_out);
    if (diag) {
        ORC_PFOR(npoin)
        for (int i = 0; i < npoin; ++i) x[i] = x[i] * d[i];
        free(d);
    }
    return st;
}

int orc_solve(int npoin, int nelem, const int *ik0, const int *ik1,
              const int *ik2, double *x, double *b, double *dm,
              char *typdia, double *xm, int ld, char typext, int slv,
              int precon, int nitmax, double eps, int dot_mode,
              int nb, int nt, int *nit_out, double *relres_out,
              int *relat_out, int krylov)
{
    opmesh M = {1, nelem, ld, ik0, ik1, ik2, 0, NULL, NULL, NULL, NULL};
    int *gptr = NULL, *gek = NULL;
    if (ORC_PAR(npoin) && build_gather(npoin, nelem, ik0, ik1, ik2, &gptr, &gek) == ORC_OK) {
        M.gptr = gptr;
        M.gek = gek;
    }
    int st = solve_impl(&M, npoin, x, b, dm, typdia, xm, typext, slv, precon, nitmax, eps,
                        krylov, dot_mode, nb, nt, nit_out, relres_out, relat_out);
    free(gptr); free(gek);
    return st;
}

/* SOLVE (SLV=1) on a segment-storage matrix (STO=3): the same algorithm with
 * MVSEG products and OMSEG scaling. */
int orc_solve_seg(int npoin, int nseg, const int *g1, const int *g2, double *x, double *b,
                  double *dm, char *typdia, double *xa, char typext, int slv, int precon,
                  int nitmax, double eps, int dot_mode, int nb, int nt, int *nit_out,
                  double *relres_out, int *relat_out, int krylov)
{
    opmesh M = {3, 0, 0, NULL, NULL, NULL, nseg, g1, g2};
    return solve_impl(&M, npoin, x, b, dm, typdia, xa, typext, slv, precon, nitmax, eps,
                      krylov, dot_mode, nb, nt, nit_out, relres_out, relat_out);
}

/* ------------------------------------------------------------------ */
/* mixed precision (no reference counterpart)                           */
/* ------------------------------------------------------------------ */

/* Node -> (element, local point) gather lists in ASSVEC order (local point
 * outer, element inner), the order in which ASSVEC adds into each node. */
static int build_gather(int npoin, int nelem, const int *ik0, const int *ik1,
                        const int *ik2, int **ptr_out, int **ek_out)
{
    int *ptr = (int *)calloc((size_t)npoin + 1, sizeof(int));
    int *ek = (int *)malloc(sizeof(int) * 3 * (size_t)nelem);
    int *pos = (int *)malloc(sizeof(int) * (size_t)npoin);
    if (!ptr || !ek || !pos) { free(ptr); free(ek); free(pos); return ORC_ERR_ARGS; }
    const int *ik[3] = {ik0, ik1, ik2};
    for (int k = 0; k < 3; ++k)
        for (int e = 0; e < nelem; ++e) ptr[ik[k][e] + 1]++;
    for (int i = 0; i < npoin; ++i) ptr[i + 1] += ptr[i];
    for (int i = 0; i < npoin; ++i) pos[i] = ptr[i];
    for (int k = 0; k < 3; ++k)
        for (int e = 0; e < nelem; ++e) ek[pos[ik[k][e]]++] = (e << 2) | k;
    free(pos);
    *ptr_out = ptr;
    *ek_out = ek;
    return ORC_OK;
}

/* Binary32 edge (segment) form of a symmetric EBE operator, built the way
 * the device builds it: for node i, scan its gather entries in ASSVEC
 * order; each entry (element e, local point k) contributes XA(k,a) to the
 * neighbour a = IKLE(e,(k+1) mod 3) and XA(k,b) to b = IKLE(e,(k+2) mod 3)
 * (the per-edge assembly ASSEX3 performs for segment storage).  Neighbours
 * get slots in order of first appearance; slot coefficients and the row sum
 * s_i = diag_i + sum of (XA(k,a) + XA(k,b)) are accumulated in binary64 in
 * scan order and rounded once to binary32. */
typedef struct {
    int npoin;
    int *nptr;    /* npoin+1: slot range of each node */
    int *col;     /* neighbour of each slot */
    float *val;   /* binary32 coefficient of each slot */
    float *s32;   /* binary32 row sums */
} seg32;

static void seg32_free(seg32 *g)
{
    free(g->nptr); free(g->col); free(g->val); free(g->s32);
}

static int seg32_build(int npoin, int nelem, const int *ik0, const int *ik1,
                       const int *ik2, const int *ptr, const int *ek,
                       const double *da, char typdia, const double *xm,
                       seg32 *g)
{
    const int *ik[3] = {ik0, ik1, ik2};
    const double *m[3] = {xm, xm + nelem, xm + 2 * (size_t)nelem};
    size_t cap = 2 * (size_t)ptr[npoin] + 1;
    g->npoin = npoin;
    g->nptr = (int *)malloc(sizeof(int) * ((size_t)npoin + 1));
    g->col = (int *)malloc(sizeof(int) * cap);
    g->val = (float *)malloc(sizeof(float) * cap);
    g->s32 = (float *)malloc(sizeof(float) * (size_t)npoin);
    double *c64 = (double *)malloc(sizeof(double) * cap);
    if (!g->nptr || !g->col || !g->val || !g->s32 || !c64) { free(c64); return ORC_ERR_ARGS; }
    size_t top = 0;
    for (int i = 0; i < npoin; ++i) {
        size_t base = top;
        g->nptr[i] = (int)base;
        double srow = typdia == 'Q' ? da[i] : (typdia == 'I' ? 1.0 : 0.0);
        for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
            int e = ek[j] >> 2, k = ek[j] & 3;
            int a = (k + 1) % 3, b = (k + 2) % 3;
            int v[2] = {ik[a][e], ik[b][e]};
            double x[2] = {m[k + a - 1][e], m[k + b - 1][e]};
            for (int q = 0; q < 2; ++q) {
                size_t sl = base;
                while (sl < top && g->col[sl] != v[q]) ++sl;
                if (sl == top) { g->col[top] = v[q]; c64[top] = 0.0; ++top; }
                c64[sl] = c64[sl] + x[q];
            }
            srow = srow + (x[0] + x[1]);
        }
        for (size_t sl = base; sl < top; ++sl) g->val[sl] = (float)c64[sl];
        g->s32[i] = (float)srow;
    }
    g->nptr[npoin] = (int)top;
    free(c64);
    return ORC_OK;
}

/* Node -> incident segment lists in ascending segment order (the order in
 * which MVSEG adds into each node): entries (ISEG<<1 | side), side 0 when
 * the node is GLOSEG1 (its term uses XA1 and Y(GLOSEG2)), 1 when GLOSEG2. */
static int build_seg_gather(int npoin, int nseg, const int *g1, const int *g2,
                            int **ptr_out, int **idx_out)
{
    int *ptr = (int *)calloc((size_t)npoin + 1, sizeof(int));
    int *idx = (int *)malloc(sizeof(int) * 2 * (size_t)nseg + 1);
    int *pos = (int *)malloc(sizeof(int) * (size_t)npoin + 1);
    if (!ptr || !idx || !pos) { free(ptr); free(idx); free(pos); return ORC_ERR_ARGS; }
    for (int sg = 0; sg < nseg; ++sg) { ptr[g1[sg] + 1]++; ptr[g2[sg] + 1]++; }
    for (int i = 0; i < npoin; ++i) ptr[i + 1] += ptr[i];
    for (int i = 0; i < npoin; ++i) pos[i] = ptr[i];
    for (int sg = 0; sg < nseg; ++sg) {
        idx[pos[g1[sg]]++] = sg << 1;
        idx[pos[g2[sg]]++] = (sg << 1) | 1;
    }
    free(pos);
    *ptr_out = ptr;
    *idx_out = idx;
    return ORC_OK;
}

/* Binary32 form of a symmetric segment operator: for node i one slot per
 * incident segment, in ascending segment order, holding the neighbour and
 * (float)XA(ISEG); the row sum s_i = diag_i + XA of each incident segment,
 * added in that order in binary64, rounded once. */
static int seg32_build_seg(int npoin, const int *g1, const int *g2, const int *ptr,
                           const int *idx, const double *da, char typdia, const double *xa,
                           seg32 *g)
{
    size_t cap = (size_t)ptr[npoin] + 1;
    g->npoin = npoin;
    g->nptr = (int *)malloc(sizeof(int) * ((size_t)npoin + 1));
    g->col = (int *)malloc(sizeof(int) * cap);
    g->val = (float *)malloc(sizeof(float) * cap);
    g->s32 = (float *)malloc(sizeof(float) * (size_t)npoin);
    if (!g->nptr || !g->col || !g->val || !g->s32) return ORC_ERR_ARGS;
    for (int i = 0; i <= npoin; ++i) g->nptr[i] = ptr[i];
    for (int i = 0; i < npoin; ++i) {
        double srow = typdia == 'Q' ? da[i] : (typdia == 'I' ? 1.0 : 0.0);
        for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
            int sg = idx[j] >> 1, side = idx[j] & 1;
            g->col[j] = side ? g1[sg] : g2[sg];
            g->val[j] = (float)xa[sg];
            srow = srow + xa[sg];
        }
        g->s32[i] = (float)srow;
    }
    return ORC_OK;
}

/* q = A32 p in difference form: q_i = s_i p_i + sum over slots of
 * c (p_j - p_i), slots in order.  Rounding the coefficients then leaves
 * constant vectors exact, so the small mass-dominated eigenvalues of the
 * wave operator survive the binary32 copy. */
static void seg32_mv(const seg32 *g, const float *p, float *q)
{
    ORC_PFOR(g->npoin)
    for (int i = 0; i < g->npoin; ++i) {
        float pi = p[i];
        float acc = pi * g->s32[i];
        for (int sl = g->nptr[i]; sl < g->nptr[i + 1]; ++sl)
            acc = acc + g->val[sl] * (p[g->col[sl]] - pi);
        q[i] = acc;
    }
}

/* Mixed-precision solve (the device kernel's exact operation order):
 * PRECD1 scaling in binary64 on copies; binary32 copy of the scaled EBE
 * operator; one binary32 CG (binary32 vectors, matvec and dots) whose
 * correction z is folded into the binary64 solution ("reliable update")
 * whenever its recursive residual has dropped by inner_tol relative to the
 * last true residual, or looks converged.  Each update recomputes the true
 * residual r = b - A x in binary64, tests it against outer_tol (relative to
 * ||b||, absolute when ||b||^2 < 1, as GRACJG), and restarts the binary32
 * residual from it while keeping the search direction (beta from the
 * recursive residual).  Symmetric storage only; inputs other than x are not
 * modified.  Returns 0 when converged, the inner iteration count when
 * max_inner or max_outer ran out, or a negative error. */
static int mixed_impl(const opmesh *M, int npoin, double *x, const double *b,
                      const double *dm_in, char typdia_in, const double *xm_in,
                      char typext, int precon, double inner_tol,
                      double outer_tol, int max_outer, int max_inner,
                      const dotspec *ds, int *outer_out, int *inner_total_out,
                      double *relres_out)
{
    if (typext != 'S') return ORC_ERR_UNSUPPORTED;
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    const int *ik0 = M->ik0, *ik1 = M->ik1, *ik2 = M->ik2;
    size_t n = (size_t)npoin, ne = (size_t)nelem;
    /* off-diagonal values: 3 per element (EBE) or 1 per segment */
    const size_t nxm = M->sto == 3 ? (size_t)M->nseg : 3 * ne;
    double *dm = (double *)malloc(sizeof(double) * n);
    double *xm = (double *)malloc(sizeof(double) * nxm + 1);
    double *bs = (double *)malloc(sizeof(double) * n);
    double *d = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * 3 * ne + 1);
    float *z = (float *)malloc(sizeof(float) * n);
    float *ri = (float *)malloc(sizeof(float) * n);
    float *p = (float *)malloc(sizeof(float) * n);
    float *q = (float *)malloc(sizeof(float) * n);
    int *gptr = NULL, *gek = NULL;
    seg32 g = {0, NULL, NULL, NULL, NULL};
    opmesh Mg = *M;
    int st = ORC_OK, outer = 0, inner = 0, diag = 0;
    double xl = 0.0, rr = 0.0, otol = 0.0;
    float rho = 0.0f, rmax = 0.0f, itol2 = 0.0f;
    char typdia = typdia_in;
    if (!dm || !xm || !bs || !d || !r || !t || !w || !z || !ri || !p || !q) {
        st = ORC_ERR_ARGS; goto done;
    }
    memcpy(dm, dm_in, sizeof(double) * n);
    memcpy(xm, xm_in, sizeof(double) * nxm);
    memcpy(bs, b, sizeof(double) * n);
    if (precon == 0) precon = 1;
    diag = (precon % 2 == 0 || precon % 3 == 0 || precon % 5 == 0);
    if (diag) {
        st = precd1_impl(M, npoin, precon, x, dm, &typdia, xm, typext, bs, d);
        if (st) goto done;
    }
    if (M->sto == 3) {
        if ((st = build_seg_gather(npoin, M->nseg, M->g1, M->g2, &gptr, &gek))) goto done;
        if ((st = seg32_build_seg(npoin, M->g1, M->g2, gptr, gek, dm, typdia, xm, &g)))
            goto done;
    } else {
        if ((st = build_gather(npoin, nelem, ik0, ik1, ik2, &gptr, &gek))) goto done;
        if ((st = seg32_build(npoin, nelem, ik0, ik1, ik2, gptr, gek, dm, typdia, xm, &g)))
            goto done;
        if (ORC_PAR(npoin)) {   /* threaded: binary64 products by the gather form */
            Mg.gptr = gptr;
            Mg.gek = gek;
        }
    }

    xl = dot64s(ds, npoin, bs, bs);
    if (sqrt(xl) < 1.0e-15) {
        for (size_t i = 0; i < n; ++i) x[i] = 0.0;
        rr = 0.0; xl = 1.0;
        goto fin;
    }
    if (xl < 1.0) xl = 1.0;
    otol = xl * (outer_tol * outer_tol);
    itol2 = (float)(inner_tol * inner_tol);

    /* true residual r = b - A x (binary64), its binary32 copy, both norms */
#define TRUE_RESIDUAL()                                                         \
    do {                                                                        \
        st = op_matvec(&Mg, "X=AY    ", npoin, t, dm, typdia, xm, typext, x, 0.0, \
                       r, w);                                                   \
        if (st) goto done;                                                      \
        ORC_PFOR(n)                                                             \
        for (size_t i = 0; i < n; ++i) { r[i] = bs[i] - t[i]; ri[i] = (float)r[i]; } \
        rr = dot64s(ds, npoin, r, r);                                          \
        rho = dot32s(ds, npoin, ri, ri);                                       \
    } while (0)

    TRUE_RESIDUAL();
    if (isnan(rr)) { st = ORC_ERR_NAN; goto fin; }
    if (rr <= otol) goto fin;
    rmax = rho;
    ORC_PFOR(n)
    for (size_t i = 0; i < n; ++i) { z[i] = 0.0f; p[i] = ri[i]; }
    for (;;) {
        seg32_mv(&g, p, q);
        float pq = dot32s(ds, npoin, p, q);
        if (!(pq > 0.0f)) { st = isnan(pq) ? ORC_ERR_NAN : ORC_ERR_BREAKDOWN; goto fin; }
        float alpha = rho / pq;
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) z[i] = z[i] + alpha * p[i];
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) ri[i] = ri[i] - alpha * q[i];
        float rho_new = dot32s(ds, npoin, ri, ri);
        float rho_rec = rho_new, rho_old = rho;
        ++inner;
        int last = inner >= max_inner;
        if (last || rho_new <= itol2 * rmax || (double)rho_new <= otol) {
            ORC_PFOR(n)
            for (size_t i = 0; i < n; ++i) { x[i] = x[i] + (double)z[i]; z[i] = 0.0f; }
            TRUE_RESIDUAL();
            ++outer;
            if (isnan(rr)) { st = ORC_ERR_NAN; goto fin; }
            if (rr <= otol) goto fin;
            if (last || outer >= max_outer) { st = inner; goto fin; }
            rho_new = rho;
            rmax = rho;
        }
        float beta = rho_rec / rho_old;
        rho = rho_new;
        ORC_PFOR(n)
        for (size_t i = 0; i < n; ++i) p[i] = ri[i] + beta * p[i];
    }
#undef TRUE_RESIDUAL
fin:
    if (diag) for (size_t i = 0; i < n; ++i) x[i] = x[i] * d[i];
    if (outer_out) *outer_out = outer;
    if (inner_total_out) *inner_total_out = inner;
    if (relres_out) *relres_out = sqrt(rr / xl);
done:
    free(dm); free(xm); free(bs); free(d); free(r); free(t); free(w);
    free(z); free(ri); free(p); free(q); free(gptr); free(gek);
    seg32_free(&g);
    return st;
}

int orc_solve_mixed(int npoin, int nelem, const int *ik0, const int *ik1,
                    const int *ik2, double *x, const double *b,
                    const double *dm_in, char typdia_in, const double *xm_in,
                    char typext, int precon, double inner_tol,
                    double outer_tol, int max_outer, int max_inner,
                    int nb, int nt, int *outer_out, int *inner_total_out,
                    double *relres_out)
{
    dotspec ds = {0, nb, nt, 1};
    opmesh M = {1, nelem, nelem, ik0, ik1, ik2, 0, NULL, NULL};
    return mixed_impl(&M, npoin, x, b, dm_in, typdia_in, xm_in,
                      typext, precon, inner_tol, outer_tol, max_outer, max_inner,
                      &ds, outer_out, inner_total_out, relres_out);
}

/* Mixed-precision solve on a segment-storage matrix (symmetric XA(NSEG)):
 * the same algorithm with the binary32 operator taken from the segments and
 * the binary64 residual from MVSEG. */
int orc_solve_mixed_seg(int npoin, int nseg, const int *g1, const int *g2, double *x,
                        const double *b, const double *dm_in, char typdia_in,
                        const double *xa_in, char typext, int precon, double inner_tol,
                        double outer_tol, int max_outer, int max_inner, int nb, int nt,
                        int *outer_out, int *inner_total_out, double *relres_out)
{
    dotspec ds = {0, nb, nt, 1};
    opmesh M = {3, 0, 0, NULL, NULL, NULL, nseg, g1, g2};
    return mixed_impl(&M, npoin, x, b, dm_in, typdia_in, xa_in, typext, precon, inner_tol,
                      outer_tol, max_outer, max_inner, &ds, outer_out, inner_total_out,
                      relres_out);
}

/* One instance of the batched solver: the same algorithm with the batched
 * kernel's dot order (nt threads per tile, npt nodes per thread). */
int orc_solve_mixed_batch(int npoin, int nelem, const int *ik0, const int *ik1,
                          const int *ik2, double *x, const double *b,
                          const double *dm_in, char typdia_in, const double *xm_in,
                          char typext, int precon, double inner_tol,
                          double outer_tol, int max_outer, int max_inner,
                          int nt, int npt, int *outer_out, int *inner_total_out,
                          double *relres_out)
{
    dotspec ds = {1, 0, nt, npt};
    opmesh M = {1, nelem, nelem, ik0, ik1, ik2, 0, NULL, NULL};
    return mixed_impl(&M, npoin, x, b, dm_in, typdia_in, xm_in,
                      typext, precon, inner_tol, outer_tol, max_outer, max_inner,
                      &ds, outer_out, inner_total_out, relres_out);
}


/* One instance of the batched solver on a segment-storage matrix: the
 * segment form of orc_solve_mixed_seg with the batched kernel's dot order. */
int orc_solve_mixed_batch_seg(int npoin, int nseg, const int *g1, const int *g2, double *x,
                              const double *b, const double *dm_in, char typdia_in,
                              const double *xa_in, char typext, int precon, double inner_tol,
                              double outer_tol, int max_outer, int max_inner, int nt, int npt,
                              int *outer_out, int *inner_total_out, double *relres_out)
{
    dotspec ds = {1, 0, nt, npt};
    opmesh M = {3, 0, 0, NULL, NULL, NULL, nseg, g1, g2, NULL, NULL};
    return mixed_impl(&M, npoin, x, b, dm_in, typdia_in, xa_in, typext, precon, inner_tol,
                      outer_tol, max_outer, max_inner, &ds, outer_out, inner_total_out,
                      relres_out);
}

/* ------------------------------------------------------------------ */
/* multi-threaded port (CPU baseline on all host cores)                 */
/* ------------------------------------------------------------------ */

/* The binary64 SOLVE/GRACJG algorithm of orc_solve on `nthreads` OpenMP
 * threads, standing in for the reference run with one MPI rank per core:
 * the matvec gathers each node's ASSVEC contributions in ASSVEC order (same
 * bits as the sequential scatter), vector updates are node-parallel, and
 * dot products sum per-thread partials of static node chunks in thread
 * order.  Symmetric storage, PRECON 2. */
static void mv_gather(int npoin, const int *ptr, const int *ek, const int *ik0,
                      const int *ik1, const int *ik2, const double *xm,
                      int nelem, char typdia, const double *da,
                      const double *y, double *out)
{
    const int *ik[3] = {ik0, ik1, ik2};
    const double *m[3] = {xm, xm + nelem, xm + 2 * (size_t)nelem};
    #pragma omp for schedule(static)
    for (int i = 0; i < npoin; ++i) {
        double acc = typdia == 'Q' ? y[i] * da[i] : (typdia == 'I' ? y[i] : 0.0);
        for (int j = ptr[i]; j < ptr[i + 1]; ++j) {
            int e = ek[j] >> 2, k = ek[j] & 3, a = (k + 1) % 3, b = (k + 2) % 3;
            acc = acc + (m[k + a - 1][e] * y[ik[a][e]] + m[k + b - 1][e] * y[ik[b][e]]);
        }
        out[i] = acc;
    }
}

static double dot_omp(int n, const double *x, const double *y, double *part)
{
    int nt = 1, t = 0;
#ifdef _OPENMP
    nt = omp_get_num_threads();
    t = omp_get_thread_num();
#endif
    double s = 0.0;
    #pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) s = s + x[i] * y[i];
    part[t] = s;
    #pragma omp barrier
    double r = 0.0;
    for (int k = 0; k < nt; ++k) r = r + part[k];
    #pragma omp barrier
    return r;
}

int orc_solve_omp(int npoin, int nelem, const int *ik0, const int *ik1,
                  const int *ik2, double *x, const double *b_in,
                  const double *dm_in, const double *xm_in, int nitmax,
                  double eps, int nthreads, int *nit_out, double *relres_out)
{
    size_t n = (size_t)npoin, ne = (size_t)nelem;
    int *ptr = NULL, *ek = NULL;
    if (build_gather(npoin, nelem, ik0, ik1, ik2, &ptr, &ek)) return ORC_ERR_ARGS;
    double *xm = (double *)malloc(sizeof(double) * 3 * ne);
    double *b = (double *)malloc(sizeof(double) * n);
    double *d = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    double *dd = (double *)malloc(sizeof(double) * n);
    double *ad = (double *)malloc(sizeof(double) * n);
    double part[1024];
    int st = ORC_OK, m_out = 0;
    double rel_out = 0.0;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
#ifdef _OPENMP
    omp_set_num_threads(nthreads);
#endif
    #pragma omp parallel
    {
        /* PRECD1 (PRECON 2) */
        #pragma omp for schedule(static)
        for (int i = 0; i < npoin; ++i) {
            double di = sqrt(dm_in[i]);
            x[i] = x[i] * di;
            di = (fabs(di) > 1.0e-10) ? 1.0 / di : 1.0;
            d[i] = di;
            b[i] = b_in[i] * di;
        }
        #pragma omp for schedule(static)
        for (int e = 0; e < nelem; ++e) {
            xm[e] = xm_in[e] * d[ik1[e]] * d[ik0[e]];
            xm[ne + e] = xm_in[ne + e] * d[ik2[e]] * d[ik0[e]];
            xm[2 * ne + e] = xm_in[2 * ne + e] * d[ik2[e]] * d[ik1[e]];
        }
        double xl = dot_omp(npoin, b, b, part), rmrm, rmgm, rm1gm1, dad, ro, beta;
        int m = 0, relat = 1;
        if (sqrt(xl) < 1.0e-15) {
            #pragma omp for schedule(static)
            for (int i = 0; i < npoin; ++i) x[i] = 0.0;
            rmrm = 0.0; xl = 1.0;
            goto fin;
        }
        if (xl < 1.0) { xl = 1.0; relat = 0; }
        (void)relat;
        mv_gather(npoin, ptr, ek, ik0, ik1, ik2, xm, nelem, 'I', NULL, x, r);
        #pragma omp for schedule(static)
        for (int i = 0; i < npoin; ++i) r[i] = r[i] - b[i];
        rmrm = dot_omp(npoin, r, r, part);
        rmgm = rmrm;
        if (rmrm < eps * eps * xl) goto fin;
        #pragma omp for schedule(static)
        for (int i = 0; i < npoin; ++i) dd[i] = r[i];
        mv_gather(npoin, ptr, ek, ik0, ik1, ik2, xm, nelem, 'I', NULL, dd, ad);
        dad = dot_omp(npoin, dd, ad, part);
        ro = rmgm / dad;
        #pragma omp for schedule(static)
        for (int i = 0; i < npoin; ++i) x[i] = x[i] + (-ro) * dd[i];
        for (;;) {
            m = m + 1;
            #pragma omp for schedule(static)
            for (int i = 0; i < npoin; ++i) r[i] = r[i] + (-ro) * ad[i];
            rm1gm1 = rmgm;
            rmrm = dot_omp(npoin, r, r, part);
            rmgm = rmrm;
            if (rmrm <= xl * (eps * eps)) break;
            beta = rmgm / rm1gm1;
            #pragma omp for schedule(static)
            for (int i = 0; i < npoin; ++i) dd[i] = r[i] + beta * dd[i];
            mv_gather(npoin, ptr, ek, ik0, ik1, ik2, xm, nelem, 'I', NULL, dd, ad);
            dad = dot_omp(npoin, dd, ad, part);
            ro = rmgm / dad;
            #pragma omp for schedule(static)
            for (int i = 0; i < npoin; ++i) x[i] = x[i] + (-ro) * dd[i];
            if (m >= nitmax) break;
        }
    fin:
        #pragma omp for schedule(static)
        for (int i = 0; i < npoin; ++i) x[i] = x[i] * d[i];
        #pragma omp single
        {
            m_out = m;
            rel_out = sqrt(rmrm / xl);
            st = (m >= nitmax && !(rmrm <= xl * (eps * eps))) ? m : ORC_OK;
        }
    }
    if (nit_out) *nit_out = m_out;
    if (relres_out) *relres_out = rel_out;
    free(ptr); free(ek); free(xm); free(b); free(d); free(r); free(dd); free(ad);
    return st;
}

/* ------------------------------------------------------------------ */
/* segment storage (STO=3)                                              */
/* ------------------------------------------------------------------ */

typedef struct { long long key; int ef; } edge_key;

static int cmp_edge(const void *a, const void *b)
{
    const edge_key *x = (const edge_key *)a, *y = (const edge_key *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->ef < y->ef ? -1 : (x->ef > y->ef);
}

/* stoseg.f:94-225 for P1 triangles with NCSIZE <= 1.  The NELEB boundary
 * segments come first, in the given order: boundary segment IELEB is face
 * nulone[IELEB] (0-based; face f joins local points f and f+1 mod 3) of
 * element nelbor[IELEB], GLOSEG = (IKLE(f), IKLE(f+1)) and ORISEG = 1
 * (:108-115).  Then every element face without a segment, elements in
 * order, faces 1..3, opens the next segment with GLOSEG ordered by node
 * number (:127-145) and gives it to the neighbour across that face
 * (IFABOR, computed here from IKLE), which must run the edge the other way
 * (:146-186).  eltseg/oriseg: 3 x nelem, face-major, 0-based segment
 * numbers, ORISEG 1 or 2.  Returns the segment count in *nseg_out. */
int orc_stoseg(int npoin, int nelem, const int *ik0, const int *ik1, const int *ik2,
               int neleb, const int *nelbor, const int *nulone, int *g1, int *g2,
               int *eltseg, int *oriseg, int *nseg_out)
{
    const int *ik[3] = {ik0, ik1, ik2};
    const int next[3] = {1, 2, 0};
    size_t nf = 3 * (size_t)nelem;
    edge_key *keys = (edge_key *)malloc(sizeof(edge_key) * nf + 1);
    int *ifabor = (int *)malloc(sizeof(int) * nf + 1);
    if (!keys || !ifabor) { free(keys); free(ifabor); return ORC_ERR_ARGS; }
    for (int f = 0; f < 3; ++f)
        for (int e = 0; e < nelem; ++e) {
            int a = ik[f][e], b = ik[next[f]][e];
            int lo = a < b ? a : b, hi = a < b ? b : a;
            keys[(size_t)f * nelem + e].key = (long long)lo * npoin + hi;
            keys[(size_t)f * nelem + e].ef = f * nelem + e;
            ifabor[(size_t)f * nelem + e] = -1;
        }
    qsort(keys, nf, sizeof(edge_key), cmp_edge);
    for (size_t q = 0; q + 1 < nf; ++q)
        if (keys[q].key == keys[q + 1].key) {
            int ea = keys[q].ef % nelem, eb = keys[q + 1].ef % nelem;
            ifabor[keys[q].ef] = eb;
            ifabor[keys[q + 1].ef] = ea;
            ++q;
        }
    free(keys);
    for (size_t q = 0; q < nf; ++q) eltseg[q] = -1;
    for (int s = 0; s < neleb; ++s) {                           /* :108-115 */
        int e = nelbor[s], f = nulone[s];
        g1[s] = ik[f][e];
        g2[s] = ik[next[f]][e];
        eltseg[(size_t)f * nelem + e] = s;
        oriseg[(size_t)f * nelem + e] = 1;
    }
    int nse = neleb, st = ORC_OK;
    for (int e1 = 0; e1 < nelem && st == ORC_OK; ++e1)          /* :119-205 */
        for (int f = 0; f < 3; ++f) {
            if (eltseg[(size_t)f * nelem + e1] >= 0) continue;
            int i1 = ik[f][e1], i2 = ik[next[f]][e1];
            if (i1 == i2) { st = ORC_ERR_BAD_MESH; break; }
            int s = nse++;
            eltseg[(size_t)f * nelem + e1] = s;
            if (i1 < i2) { g1[s] = i1; g2[s] = i2; oriseg[(size_t)f * nelem + e1] = 1; }
            else { g1[s] = i2; g2[s] = i1; oriseg[(size_t)f * nelem + e1] = 2; }
            int e2 = ifabor[(size_t)f * nelem + e1];
            if (e2 < 0) continue;
            int found = 0;
            for (int jf = 0; jf < 3; ++jf) {
                int j1 = ik[jf][e2], j2 = ik[next[jf]][e2];
                if (i1 == j2 && i2 == j1) {
                    eltseg[(size_t)jf * nelem + e2] = s;
                    oriseg[(size_t)jf * nelem + e2] = 3 - oriseg[(size_t)f * nelem + e1];
                    found = 1;
                    break;
                } else if (i1 == j1 && i2 == j2) {
                    break;                                      /* wrongly oriented */
                }
            }
            if (!found) { st = ORC_ERR_BAD_MESH; break; }
        }
    free(ifabor);
    *nseg_out = nse;
    return st;
}

/* assex3.f:150-160 -> as3_1111_s.f:71-79 ('S') and as3_1111_q.f:85-98
 * ('Q', STOXMT=1): EBE off-diagonal terms summed into segments, element by
 * element, from zero.  Face 1 (points 1-2) takes XMT(,1) [and XMT(,4)],
 * face 2 (2-3) XMT(,3) [and XMT(,6)], face 3 (3-1) XMT(,2) [XMT(,5)]; for
 * 'Q' the term of row IKLE(f) goes to column ORISEG of XA(NSEG,2) and the
 * other to column 3-ORISEG.  xmt: ld x (3|6) column-major. */
int orc_assex3(int nelem, const int *eltseg, const int *oriseg, char typext,
               const double *xmt, int ld, int nseg, double *xa)
{
    const double *m[6];
    for (int c = 0; c < 6; ++c) m[c] = xmt + (size_t)c * ld;
    const int *es1 = eltseg, *es2 = eltseg + nelem, *es3 = eltseg + 2 * (size_t)nelem;
    if (typext == 'S') {
        for (int s = 0; s < nseg; ++s) xa[s] = 0.0;
        for (int e = 0; e < nelem; ++e) {
            xa[es1[e]] = xa[es1[e]] + m[0][e];
            xa[es2[e]] = xa[es2[e]] + m[2][e];
            xa[es3[e]] = xa[es3[e]] + m[1][e];
        }
        return ORC_OK;
    }
    if (typext != 'Q') return ORC_ERR_ARGS;
    const int *o1 = oriseg, *o2 = oriseg + nelem, *o3 = oriseg + 2 * (size_t)nelem;
    double *x1 = xa, *x2 = xa + nseg;
#define XA(s, o) (*((o) == 1 ? &x1[s] : &x2[s]))
    for (int s = 0; s < nseg; ++s) { x1[s] = 0.0; x2[s] = 0.0; }
    for (int e = 0; e < nelem; ++e) {
        XA(es1[e], o1[e]) = XA(es1[e], o1[e]) + m[0][e];
        XA(es2[e], o2[e]) = XA(es2[e], o2[e]) + m[2][e];
        XA(es3[e], o3[e]) = XA(es3[e], o3[e]) + m[4][e];
        XA(es1[e], 3 - o1[e]) = XA(es1[e], 3 - o1[e]) + m[3][e];
        XA(es2[e], 3 - o2[e]) = XA(es2[e], 3 - o2[e]) + m[5][e];
        XA(es3[e], 3 - o3[e]) = XA(es3[e], 3 - o3[e]) + m[1][e];
    }
#undef XA
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Dirichlet conditions                                                 */
/* ------------------------------------------------------------------ */

/* diri01.f:90-130 with boundary values (FBOR on the NPTFR boundary points,
 * DIRAUX diraux.f:70-85 on boundary numbering): W1 = 0, W1(NBOR(K)) = FBOR(K)
 * where LIMDIR(K) = KDIR (OSDBIF 'X=Y'); W2 = S W1 (MATVEC 'X=AY'); SM = SM -
 * W2; W2 = 1; for those K, N = NBOR(K): SM(N) = S%D(N)*FBOR(K), W2(N) = 0,
 * F(N) = FBOR(K); with a mask SM, F and W2 are multiplied by MASKPT; then
 * OM 'M=DMD' with D = W2 on the off-diagonal terms only (TYPDIA set to '0'
 * around the call), which zeroes the rows and columns of the Dirichlet
 * points.  nbor is 0-based. */
static int diri01_impl(const opmesh *M, int npoin, const double *dm, char typdia, double *xm,
                       char typext, int nptfr, const int *nbor, const int *limdir, int kdir,
                       const double *fbor, double *sm, double *f, const double *maskpt)
{
    const int nelem = M->sto == 3 ? 0 : M->nelem;
    double *w1 = (double *)calloc((size_t)npoin, sizeof(double));
    double *w2 = (double *)malloc(sizeof(double) * (size_t)npoin);
    double *t = (double *)malloc(sizeof(double) * (size_t)npoin);
    double *w = (double *)malloc(sizeof(double) * 3 * (size_t)nelem + 1);
    int st = ORC_OK;
    if (!w1 || !w2 || !t || !w) { st = ORC_ERR_ARGS; goto done; }
    for (int k = 0; k < nptfr; ++k)
        if (limdir[k] == kdir) w1[nbor[k]] = fbor[k];
    st = op_matvec(M, "X=AY    ", npoin, w2, dm, typdia, xm, typext, w1, 0.0, t, w);
    if (st) goto done;
    for (int i = 0; i < npoin; ++i) sm[i] = sm[i] - w2[i];
    for (int i = 0; i < npoin; ++i) w2[i] = 1.0;
    for (int k = 0; k < nptfr; ++k)
        if (limdir[k] == kdir) {
            int n = nbor[k];
            sm[n] = dm[n] * fbor[k];
            w2[n] = 0.0;
            f[n] = fbor[k];
        }
    if (maskpt)
        for (int i = 0; i < npoin; ++i) {
            sm[i] = sm[i] * maskpt[i];
            f[i] = f[i] * maskpt[i];
            w2[i] = w2[i] * maskpt[i];
        }
    {
        /* OM 'M=DMD' with TYPDIA '0': off-diagonal part only (omseg.f:530-541,
         * om1111.f:589-600) */
        const double *dsc = w2;
        if (M->sto == 3) {
            if (typext == 'S' || typext == 'Q') {
                for (int s = 0; s < M->nseg; ++s) xm[s] = xm[s] * dsc[M->g1[s]] * dsc[M->g2[s]];
                if (typext == 'Q')
                    for (int s = 0; s < M->nseg; ++s)
                        xm[M->nseg + s] = xm[M->nseg + s] * dsc[M->g1[s]] * dsc[M->g2[s]];
            }
        } else if (typext == 'S' || typext == 'Q') {
            const int ld = M->ld;
            const int *ik0 = M->ik0, *ik1 = M->ik1, *ik2 = M->ik2;
            double *x1 = xm, *x2 = xm + ld, *x3 = xm + 2 * (size_t)ld;
            for (int e = 0; e < nelem; ++e) {
                x1[e] = x1[e] * dsc[ik1[e]] * dsc[ik0[e]];
                x2[e] = x2[e] * dsc[ik2[e]] * dsc[ik0[e]];
                x3[e] = x3[e] * dsc[ik2[e]] * dsc[ik1[e]];
            }
            if (typext == 'Q') {
                double *x4 = xm + 3 * (size_t)ld, *x5 = xm + 4 * (size_t)ld,
                       *x6 = xm + 5 * (size_t)ld;
                for (int e = 0; e < nelem; ++e) {
                    x4[e] = x4[e] * dsc[ik1[e]] * dsc[ik0[e]];
                    x5[e] = x5[e] * dsc[ik2[e]] * dsc[ik0[e]];
                    x6[e] = x6[e] * dsc[ik2[e]] * dsc[ik1[e]];
                }
            }
        }
    }
done:
    free(w1); free(w2); free(t); free(w);
    return st;
}

int orc_diri01(int npoin, int nelem, const int *ik0, const int *ik1, const int *ik2,
               const double *dm, char typdia, double *xm, char typext, int nptfr,
               const int *nbor, const int *limdir, int kdir, const double *fbor, double *sm,
               double *f, const double *maskpt)
{
    opmesh M = {1, nelem, nelem, ik0, ik1, ik2, 0, NULL, NULL};
    return diri01_impl(&M, npoin, dm, typdia, xm, typext, nptfr, nbor, limdir, kdir, fbor, sm,
                       f, maskpt);
}

int orc_diri01_seg(int npoin, int nseg, const int *g1, const int *g2, const double *dm,
                   char typdia, double *xa, char typext, int nptfr, const int *nbor,
                   const int *limdir, int kdir, const double *fbor, double *sm, double *f,
                   const double *maskpt)
{
    opmesh M = {3, 0, 0, NULL, NULL, NULL, nseg, g1, g2};
    return diri01_impl(&M, npoin, dm, typdia, xa, typext, nptfr, nbor, limdir, kdir, fbor, sm,
                       f, maskpt);
}
