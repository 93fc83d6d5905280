/*
 * CPU oracle for the FRiBoIS2D fluid time step -- TEST INFRASTRUCTURE ONLY.
 * See fbo.h for scope and parity status ("parity unpinned" against the
 * Fortran binary; LAPACK pieces pinned against scipy's LAPACK by the tests).
 *
 * Every function restates one reference routine, cited by file:line, with
 * the same loop order and the same left-to-right operation order; compile
 * with -ffp-contract=off so that no multiply-add is fused (the reference is
 * built -O3 -msse2, which has no FMA).  OpenMP is used only over independent
 * lines/columns; reductions stay sequential so results do not depend on the
 * thread count.
 */
#include "fbo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KG 2 /* ghost rows below k = 1 kept: the reference allocates kstart-3 */

struct fbo_state {
    fbo_params p;
    int n2, n3, n2m, n3m, nlm, status;
    double dx2, dx3, dx2q, dx3q, ren, pi;
    double gam[3], rom[3], alm[3];
    double al, ga, ro, beta, dt, dt_o, time, cflm, q3avg, nbcv, nbcw, ddmin, pravg;
    /* 1-D grid data, 1-based */
    double *rc, *rm, *zz, *zm, *g2rc, *g2rm, *g3rc, *g3rm, *udx2c, *udx2m, *udx3c, *udx3m;
    int *jmv, *jpv, *jmc, *jpc, *kmv, *kpv, *kmc, *kpc;
    double *am2j, *ac2j, *ap2j, *am3j, *ac3j, *ap3j;
    double *am3ck, *ac3ck, *ap3ck, *am3sk, *ac3sk, *ap3sk;
    double *amphj, *acphj, *apphj, *amphk, *acphk, *apphk;
    double *wr, *zmm, *zmmt; /* n3m, n3m x n3m column-major */
    /* fields, column-major (j, k), k = -2..n3+2 */
    double *q2, *q3, *pr, *dph, *q2f, *q3f, *rhs, *rhs2, *rhs3, *ru2, *ru3, *qcap, *fey, *fez;
    double *hmn, *vmn; /* Poisson work */
    /* inflow / outflow, 1-based n2 */
    double *qb2s, *qb2n, *dqb2s, *dqb2n, *qb3s, *qb3n, *dqb3s, *dqb3n, *dq2x2o, *dq3x2o;
    /* markers */
    double *lmcc, *lmvel, *lmacc, *lmnor, *lmA, *vert;
    int *lmind, *eulins;
    double *phi, *cl, *press, *tau, *bcerrv, *bcerrw;
    /* rigid body */
    double rigid[18]; /* cmp_n, cmv_n, cma_n, cmp_np1, cmv_np1, cma_np1 */
    double kinori[3][3];
    double forces[8];
    double scalars[13];
    double *snap; /* saved start-of-step state of the coupling iteration */
};

#define FLD(a, j, k) (a)[(size_t)((k) + KG) * (size_t)n2 + (size_t)((j) - 1)]
#define M2(a, i, d) (a)[((size_t)(i) - 1) * 2 + ((d) - 1)]
#define LMIND(i, idir, c) s->lmind[(((i) - 1) * 2 + ((idir) - 1)) * 2 + ((c) - 1)]
#define EULINS(i, idir, c, m) s->eulins[((((i) - 1) * 2 + ((idir) - 1)) * 2 + ((c) - 1)) * 9 + ((m) - 1)]
#define PHI(i, idir, m) s->phi[(((i) - 1) * 2 + ((idir) - 1)) * 9 + ((m) - 1)]
#define CL(i, idir) s->cl[((i) - 1) * 2 + ((idir) - 1)]
#define CMP_N (s->rigid + 0)
#define CMV_N (s->rigid + 3)
#define CMA_N (s->rigid + 6)
#define CMP_NP1 (s->rigid + 9)
#define CMV_NP1 (s->rigid + 12)
#define CMA_NP1 (s->rigid + 15)

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }
static int *ialloc(size_t n) { return (int *)calloc(n ? n : 1, sizeof(int)); }
static double dmax(double a, double b) { return a > b ? a : b; }

void fbo_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ LAPACK */

/* DGTTRF (LAPACK 3.8): LU of a tridiagonal matrix with partial pivoting.
 * dl, du: n-1; d: n; du2: n-2; ipiv 1-based.  Arrays here are 0-based. */
int fbo_dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv)
{
    int i;
    double fact, temp;
    if (n <= 0) return 0;
    for (i = 0; i < n; i++) ipiv[i] = i + 1;
    for (i = 0; i < n - 2; i++) du2[i] = 0.0;
    for (i = 0; i < n - 2; i++) {
        if (fabs(d[i]) >= fabs(dl[i])) {
            if (d[i] != 0.0) {
                fact = dl[i] / d[i];
                dl[i] = fact;
                d[i + 1] = d[i + 1] - fact * du[i];
            }
        } else {
            fact = d[i] / dl[i];
            d[i] = dl[i];
            dl[i] = fact;
            temp = du[i];
            du[i] = d[i + 1];
            d[i + 1] = temp - fact * d[i + 1];
            du2[i] = du[i + 1];
            du[i + 1] = -fact * du[i + 1];
            ipiv[i] = i + 2;
        }
    }
    if (n > 1) {
        i = n - 2;
        if (fabs(d[i]) >= fabs(dl[i])) {
            if (d[i] != 0.0) {
                fact = dl[i] / d[i];
                dl[i] = fact;
                d[i + 1] = d[i + 1] - fact * du[i];
            }
        } else {
            fact = d[i] / dl[i];
            d[i] = dl[i];
            dl[i] = fact;
            temp = du[i];
            du[i] = d[i + 1];
            d[i + 1] = temp - fact * d[i + 1];
            ipiv[i] = i + 2;
        }
    }
    for (i = 0; i < n; i++)
        if (d[i] == 0.0) return i + 1;
    return 0;
}

/* DGTTRS -> DGTTS2, one right-hand side, no transpose (LAPACK 3.8). */
void fbo_dgtts2(int n, const double *dl, const double *d, const double *du, const double *du2,
                const int *ipiv, double *b)
{
    int i;
    if (n <= 0) return;
    for (i = 0; i < n - 1; i++) {
        int ip = ipiv[i] - 1; /* 0-based row that was pivoted into row i */
        double temp = b[i + 1 - ip + i] - dl[i] * b[ip];
        b[i] = b[ip];
        b[i + 1] = temp;
    }
    b[n - 1] = b[n - 1] / d[n - 1];
    if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
    for (i = n - 3; i >= 0; i--) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];
}

/* full system (sub-, diagonal, super-diagonal as the reference slices them):
 * am[0..n-2] = lower(2:n), ac[0..n-1], ap[0..n-2] = upper(1:n-1) */
static void tri_solve(int n, double *am, double *ac, double *ap, double *b, double *du2, int *ipiv)
{
    fbo_dgttrf(n, am, ac, ap, du2, ipiv);
    fbo_dgtts2(n, am, ac, ap, du2, ipiv, b);
}

/* ------------------------------------------------------------------ set-up */

/* indic.F90:266-306 */
static void indic(fbo_state *s)
{
    int n2 = s->n2, n3m = s->n3m, n2m = s->n2m, kc, jc;
    for (kc = 1; kc <= n3m; kc++) {
        s->kmv[kc] = kc - 1;
        s->kpv[kc] = kc + 1;
        if (kc == 1) s->kmv[kc] = kc;
        if (kc == n3m) s->kpv[kc] = kc;
    }
    for (kc = 1; kc <= n3m; kc++) {
        s->kpc[kc] = s->kpv[kc] - kc;
        s->kmc[kc] = kc - s->kmv[kc];
    }
    for (jc = 1; jc <= n2; jc++) {
        s->jmv[jc] = jc - 1;
        s->jpv[jc] = jc + 1;
        if (jc == 1) s->jmv[jc] = jc;
        if (jc == n2m) s->jpv[jc] = jc;
        if (jc == n2) s->jpv[jc] = jc;
    }
    for (jc = 1; jc <= n2m; jc++) {
        s->jpc[jc] = s->jpv[jc] - jc;
        s->jmc[jc] = jc - s->jmv[jc];
    }
}

/* cordin.F90:105-233 with istr2 = istr3 = 100 (grid read from file) */
static void cordin(fbo_state *s)
{
    int n2 = s->n2, n3 = s->n3, n2m = s->n2m, n3m = s->n3m, j, k, i;
    double dymin, dzmin, tmp;
    for (j = 1; j <= n2m; j++) {
        s->rm[j] = (s->rc[j] + s->rc[j + 1]) * 0.5;
        s->g2rm[j] = (s->rc[j + 1] - s->rc[j]) * s->dx2;
    }
    for (j = 2; j <= n2m; j++) s->g2rc[j] = (s->rc[j + 1] - s->rc[j - 1]) * s->dx2 * 0.5;
    s->g2rc[1] = (s->rc[2] - s->rc[1]) * s->dx2;
    s->g2rc[n2] = (s->rc[n2] - s->rc[n2m]) * s->dx2;
    s->rm[n2] = s->rc[n2];
    for (j = 1; j <= n2m; j++) {
        s->udx2m[j] = s->dx2 / s->g2rm[j];
        s->udx2c[j] = s->dx2 / s->g2rc[j];
    }
    s->udx2c[n2] = s->dx2 / s->g2rc[n2];

    for (k = 1; k <= n3m; k++) {
        s->zm[k] = (s->zz[k] + s->zz[k + 1]) * 0.5;
        s->g3rm[k] = (s->zz[k + 1] - s->zz[k]) * s->dx3;
    }
    for (k = 2; k <= n3m; k++) s->g3rc[k] = (s->zz[k + 1] - s->zz[k - 1]) * s->dx3 * 0.5;
    s->g3rc[1] = (s->zz[2] - s->zz[1]) * s->dx3;
    s->g3rc[n3] = (s->zz[n3] - s->zz[n3m]) * s->dx3;
    s->zm[n3] = s->zz[n3];
    for (k = 1; k <= n3m; k++) {
        s->udx3m[k] = s->dx3 / s->g3rm[k];
        s->udx3c[k] = s->dx3 / s->g3rc[k];
    }
    s->udx3c[n3] = s->dx3 / s->g3rc[n3];

    dymin = 1.0e+6;
    for (i = 2; i <= n2; i++) {
        tmp = s->rc[i] - s->rc[i - 1];
        dymin = fmin(dymin, tmp);
    }
    dzmin = 1.0e+6;
    for (i = 2; i <= n3; i++) {
        tmp = s->zz[i] - s->zz[i - 1];
        dzmin = fmin(dzmin, tmp);
    }
    s->ddmin = fmin(dzmin, dymin);
    s->ddmin = s->ddmin * s->p.kprobe;
}

/* coetar.F90:284-423 */
static void coetar(fbo_state *s)
{
    int n2 = s->n2, n3 = s->n3, n2m = s->n2m, n3m = s->n3m;
    int kc, jc, km, kp, jm, jp;
    double a33, a33m, a33p, a22, a22m, a22p;
    double inwn = s->p.inslwn ? 1.0 : 0.0, inws = s->p.inslws ? 1.0 : 0.0;
    double dx2q = s->dx2q, dx3q = s->dx3q;

    s->am2j[1] = 0.0; s->ap2j[1] = 0.0; s->ac2j[1] = 1.0;
    s->am2j[n2] = 0.0; s->ap2j[n2] = 0.0; s->ac2j[n2] = 1.0;
    for (jc = 2; jc <= n2m; jc++) {
        jm = jc - 1;
        a22 = dx2q / s->g2rc[jc];
        a22p = 1.0 / s->g2rm[jc];
        a22m = 1.0 / s->g2rm[jm];
        s->ap2j[jc] = a22 * a22p;
        s->am2j[jc] = a22 * a22m;
        s->ac2j[jc] = -(a22 * a22p + a22 * a22m);
    }
    for (jc = 2; jc <= n2m - 1; jc++) {
        jp = s->jpv[jc];
        a22 = dx2q / s->g2rm[jc];
        a22p = a22 / s->g2rc[jp];
        a22m = a22 / s->g2rc[jc];
        s->ap3j[jc] = a22p;
        s->am3j[jc] = a22m;
        s->ac3j[jc] = -(a22p + a22m);
    }
    jc = n2m;
    jp = jc + 1;
    a22 = dx2q / s->g2rm[jc];
    a22p = +a22 / s->g2rc[jp];
    a22m = +a22 / s->g2rc[jc];
    s->am3j[jc] = a22m;
    s->ap3j[jc] = 2.0 * inwn * a22p;
    s->ac3j[jc] = -(a22m + inwn * a22p * 2.0);
    jc = 1;
    jp = jc + 1;
    a22 = dx2q / s->g2rm[jc];
    a22p = +a22 / s->g2rc[jp];
    a22m = +a22 / s->g2rc[jc];
    s->ap3j[jc] = a22p;
    s->am3j[jc] = 2.0 * a22m * inws;
    s->ac3j[jc] = -(a22p + 2.0 * inws * a22m);

    s->am3ck[1] = 0.0; s->ap3ck[1] = 0.0; s->ac3ck[1] = 1.0;
    s->am3ck[n3] = 0.0; s->ap3ck[n3] = 0.0; s->ac3ck[n3] = 1.0;
    for (kc = 2; kc <= n3m; kc++) {
        km = kc - 1;
        kp = kc + 1;
        a33 = dx3q / s->g3rc[kc];
        a33p = 1.0 / s->g3rm[kc];
        a33m = 1.0 / s->g3rm[km];
        s->ap3ck[kc] = a33 * a33p;
        s->am3ck[kc] = a33 * a33m;
        s->ac3ck[kc] = -(s->ap3ck[kc] + s->am3ck[kc]);
        (void)kp;
    }
    for (kc = 2; kc <= n3m - 1; kc++) {
        kp = kc + 1;
        a33 = dx3q / s->g3rm[kc];
        a33p = +a33 / s->g3rc[kp];
        a33m = +a33 / s->g3rc[kc];
        s->ap3sk[kc] = a33p;
        s->am3sk[kc] = a33m;
        s->ac3sk[kc] = -(s->ap3sk[kc] + s->am3sk[kc]);
    }
    kc = 1;
    kp = kc + 1;
    a33 = dx3q / s->g3rm[kc];
    a33p = +a33 / s->g3rc[kp];
    a33m = +a33 / s->g3rc[kc];
    s->ap3sk[kc] = a33p;
    s->am3sk[kc] = 0.0;
    s->ac3sk[kc] = -(a33p + a33m * 2.0);
    kc = n3m;
    kp = kc + 1;
    a33 = dx3q / s->g3rm[kc];
    a33p = +a33 / s->g3rc[kp];
    a33m = +a33 / s->g3rc[kc];
    s->am3sk[kc] = a33m;
    s->ap3sk[kc] = 0.0;
    s->ac3sk[kc] = -(a33m + a33p * 2.0);
}

/* phini.F90:109-145 (tridiag_matrices) */
static void tridiag_matrices(fbo_state *s)
{
    int n2m = s->n2m, n3m = s->n3m, jc, jp, kc, kp;
    double ugmmm, a33icc, a33icp, a22icc, a22icp;
    for (jc = 1; jc <= n2m; jc++) {
        jp = s->jpv[jc];
        a22icc = (double)s->jmc[jc] * s->dx2q / s->g2rc[jc];
        a22icp = (double)s->jpc[jc] * s->dx2q / s->g2rc[jp];
        ugmmm = 1.0 / s->g2rm[jc];
        s->amphj[jc] = a22icc * ugmmm;
        s->apphj[jc] = a22icp * ugmmm;
        s->acphj[jc] = -(s->amphj[jc] + s->apphj[jc]);
    }
    for (kc = 1; kc <= n3m; kc++) {
        kp = s->kpv[kc];
        a33icc = (double)s->kmc[kc] * s->dx3q / s->g3rc[kc];
        a33icp = (double)s->kpc[kc] * s->dx3q / s->g3rc[kp];
        ugmmm = 1.0 / s->g3rm[kc];
        s->amphk[kc] = a33icc * ugmmm;
        s->apphk[kc] = a33icp * ugmmm;
        s->acphk[kc] = -(s->amphk[kc] + s->apphk[kc]);
    }
}

/* rigid.F90:468-495 */
static void createnorm(int nlm, const double *vert, double orient, double *norm)
{
    int i;
    for (i = 1; i <= nlm; i++) {
        double t[9], v1[3], v2[3], c[3], den;
        t[0] = 0.0; t[1] = M2(vert, i, 1); t[2] = M2(vert, i, 2);
        t[3] = 0.0; t[4] = M2(vert, i + 1, 1); t[5] = M2(vert, i + 1, 2);
        t[6] = orient;
        t[7] = (M2(vert, i, 1) + M2(vert, i + 1, 1)) * 0.5;
        t[8] = (M2(vert, i, 2) + M2(vert, i + 1, 2)) * 0.5;
        v1[0] = t[3] - t[0]; v1[1] = t[4] - t[1]; v1[2] = t[5] - t[2];
        v2[0] = t[6] - t[0]; v2[1] = t[7] - t[1]; v2[2] = t[8] - t[2];
        /* utils_math.f90:51-63 */
        c[0] = v1[1] * v2[2] - v1[2] * v2[1];
        c[1] = v1[2] * v2[0] - v1[0] * v2[2];
        c[2] = v1[0] * v2[1] - v1[1] * v2[0];
        den = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        c[0] = c[0] / den; c[1] = c[1] / den; c[2] = c[2] / den;
        M2(norm, i, 1) = c[1];
        M2(norm, i, 2) = c[2];
    }
}

/* rigid.F90:142-161 */
static void get_rotmat(double a, double r[2][2])
{
    r[0][0] = cos(a);
    r[0][1] = -sin(a);
    r[1][0] = sin(a);
    r[1][1] = cos(a);
}

/* utils_proc.F90:519-578 (markers from vertices) and rigid_pre.F90:4-140 */
static void rigid_setup(fbo_state *s)
{
    int i, nlm = s->nlm;
    double r[2][2];
    for (i = 1; i <= nlm; i++) {
        double dy, dz;
        M2(s->lmcc, i, 1) = (M2(s->vert, i, 1) + M2(s->vert, i + 1, 1)) * 0.5;
        M2(s->lmcc, i, 2) = (M2(s->vert, i, 2) + M2(s->vert, i + 1, 2)) * 0.5;
        dy = M2(s->vert, i + 1, 1) - M2(s->vert, i, 1);
        dz = M2(s->vert, i + 1, 2) - M2(s->vert, i, 2);
        s->lmA[i - 1] = sqrt(dy * dy + dz * dz);
    }
    createnorm(nlm, s->vert, -1.0, s->lmnor);

    CMP_N[0] = s->p.cmposi[0];
    CMP_N[1] = s->p.cmposi[1];
    CMP_N[2] = s->p.cmroti;
    for (i = 0; i < 3; i++) CMV_N[i] = CMA_N[i] = 0.0;
    s->kinori[0][0] = s->p.cmposi[0];
    s->kinori[0][1] = s->p.cmposi[1];
    s->kinori[0][2] = s->p.cmroti;
    for (i = 0; i < 3; i++) s->kinori[1][i] = CMV_N[i], s->kinori[2][i] = CMA_N[i];
    /* ipert is read into a scalar dummy (utils_proc.F90:12,25): only the
     * first value reaches cmv_n */
    CMV_N[0] = s->p.ipert[0];
    CMV_N[1] = 0.0;
    CMV_N[2] = 0.0;
    if (s->p.rtcoup) CMV_N[2] = CMV_N[0] / s->p.rrr;
    for (i = 0; i < 3; i++) {
        CMP_NP1[i] = CMP_N[i];
        CMV_NP1[i] = CMV_N[i];
        CMA_NP1[i] = CMA_N[i];
    }
    get_rotmat(CMP_N[2], r);
    for (i = 1; i <= nlm; i++) {
        double rho[2], posP[2], velP[2], accP[2], c1[2], c2[2], c3[2];
        rho[0] = M2(s->lmcc, i, 1) - CMP_N[0];
        rho[1] = M2(s->lmcc, i, 2) - CMP_N[1];
        posP[0] = CMP_NP1[0] + (r[0][0] * rho[0] + r[0][1] * rho[1]);
        posP[1] = CMP_NP1[1] + (r[1][0] * rho[0] + r[1][1] * rho[1]);
        c1[0] = -CMV_NP1[2] * rho[1];
        c1[1] = CMV_NP1[2] * rho[0];
        velP[0] = CMV_NP1[0] + c1[0];
        velP[1] = CMV_NP1[1] + c1[1];
        c2[0] = -CMA_NP1[2] * rho[1];
        c2[1] = CMA_NP1[2] * rho[0];
        c3[0] = -CMV_NP1[2] * c1[1];
        c3[1] = CMV_NP1[2] * c1[0];
        accP[0] = CMA_NP1[0] + c2[0] + c3[0];
        accP[1] = CMA_NP1[1] + c2[1] + c3[1];
        M2(s->lmcc, i, 1) = posP[0]; M2(s->lmcc, i, 2) = posP[1];
        M2(s->lmvel, i, 1) = velP[0]; M2(s->lmvel, i, 2) = velP[1];
        M2(s->lmacc, i, 1) = accP[0]; M2(s->lmacc, i, 2) = accP[1];
    }
    for (i = 1; i <= nlm + 1; i++) {
        double rad[2];
        rad[0] = M2(s->vert, i, 1) - s->p.cmposi[0];
        rad[1] = M2(s->vert, i, 2) - s->p.cmposi[1];
        M2(s->vert, i, 1) = CMP_NP1[0] + (r[0][0] * rad[0] + r[0][1] * rad[1]);
        M2(s->vert, i, 2) = CMP_NP1[1] + (r[1][0] * rad[0] + r[1][1] * rad[1]);
    }
    createnorm(nlm, s->vert, -1.0, s->lmnor);
}

fbo_state *fbo_create(const fbo_params *p, const double *ycoord, const double *zcoord,
                      const double *vert)
{
    fbo_state *s = (fbo_state *)calloc(1, sizeof(fbo_state));
    int n2, n3, k, j, nlm;
    size_t nf;
    s->p = *p;
    n2 = s->n2 = p->n2;
    n3 = s->n3 = p->n3;
    s->n2m = n2 - 1;
    s->n3m = n3 - 1;
    nlm = s->nlm = p->nlm;
    /* fluid_pre.F90:135-182 */
    s->dx2 = 1.0 / (p->rext2 / (double)s->n2m);
    s->dx3 = 1.0 / (p->alx3 / (double)s->n3m);
    s->dx2q = s->dx2 * s->dx2;
    s->dx3q = s->dx3 * s->dx3;
    s->ren = 1.0 / p->visc;
    s->pi = 2.0 * asin(1.0);
    if (p->nsst > 1) {
        s->gam[0] = 8.0 / 15.0; s->gam[1] = 5.0 / 12.0; s->gam[2] = 3.0 / 4.0;
        s->rom[0] = 0.0; s->rom[1] = -17.0 / 60.0; s->rom[2] = -5.0 / 12.0;
    } else {
        s->gam[0] = 1.5; s->gam[1] = 0.0; s->gam[2] = 0.0;
        s->rom[0] = -0.50; s->rom[1] = 0.0; s->rom[2] = 0.0;
    }
    for (k = 0; k < p->nsst; k++) s->alm[k] = s->gam[k] + s->rom[k];
    s->dt = p->dt;
    s->dt_o = p->dt;
    s->time = 0.0;

#define A1(x, n) s->x = dalloc((size_t)(n) + 2)
#define I1(x, n) s->x = ialloc((size_t)(n) + 2)
    A1(rc, n2); A1(rm, n2); A1(zz, n3); A1(zm, n3);
    A1(g2rc, n2); A1(g2rm, n2); A1(g3rc, n3); A1(g3rm, n3);
    A1(udx2c, n2); A1(udx2m, n2); A1(udx3c, n3); A1(udx3m, n3);
    I1(jmv, n2); I1(jpv, n2); I1(jmc, n2); I1(jpc, n2);
    I1(kmv, n3); I1(kpv, n3); I1(kmc, n3); I1(kpc, n3);
    A1(am2j, n2); A1(ac2j, n2); A1(ap2j, n2); A1(am3j, n2); A1(ac3j, n2); A1(ap3j, n2);
    A1(am3ck, n3); A1(ac3ck, n3); A1(ap3ck, n3); A1(am3sk, n3); A1(ac3sk, n3); A1(ap3sk, n3);
    A1(amphj, n2); A1(acphj, n2); A1(apphj, n2); A1(amphk, n3); A1(acphk, n3); A1(apphk, n3);
    A1(qb2s, n2); A1(qb2n, n2); A1(dqb2s, n2); A1(dqb2n, n2);
    A1(qb3s, n2); A1(qb3n, n2); A1(dqb3s, n2); A1(dqb3n, n2);
    A1(dq2x2o, n2); A1(dq3x2o, n2);
#undef A1
#undef I1
    s->wr = dalloc((size_t)s->n3m);
    s->zmm = dalloc((size_t)s->n3m * s->n3m);
    s->zmmt = dalloc((size_t)s->n3m * s->n3m);
    nf = (size_t)n2 * (size_t)(n3 + 1 + 2 * KG);
    s->q2 = dalloc(nf); s->q3 = dalloc(nf); s->pr = dalloc(nf); s->dph = dalloc(nf);
    s->q2f = dalloc(nf); s->q3f = dalloc(nf); s->rhs = dalloc(nf); s->rhs2 = dalloc(nf);
    s->rhs3 = dalloc(nf); s->ru2 = dalloc(nf); s->ru3 = dalloc(nf); s->qcap = dalloc(nf);
    s->fey = dalloc(nf); s->fez = dalloc(nf);
    s->hmn = dalloc((size_t)s->n2m * s->n3m);
    s->vmn = dalloc((size_t)s->n2m * s->n3m);

    s->lmcc = dalloc((size_t)nlm * 2); s->lmvel = dalloc((size_t)nlm * 2);
    s->lmacc = dalloc((size_t)nlm * 2); s->lmnor = dalloc((size_t)nlm * 2);
    s->lmA = dalloc((size_t)nlm); s->vert = dalloc((size_t)(nlm + 1) * 2);
    s->lmind = ialloc((size_t)nlm * 4); s->eulins = ialloc((size_t)nlm * 36);
    s->phi = dalloc((size_t)nlm * 18); s->cl = dalloc((size_t)nlm * 2);
    s->press = dalloc((size_t)nlm); s->tau = dalloc((size_t)nlm * 2);
    s->bcerrv = dalloc((size_t)nlm); s->bcerrw = dalloc((size_t)nlm);

    for (j = 1; j <= n2; j++) s->rc[j] = ycoord[j - 1];
    for (k = 1; k <= n3; k++) s->zz[k] = zcoord[k - 1];
    indic(s);
    cordin(s);
    tridiag_matrices(s);

    /* inqpr, initial_sol.F90:251-299 (k = kstart-1 .. kend+1) */
    for (k = 0; k <= n3; k++)
        for (j = 1; j <= n2; j++) {
            FLD(s->q2, j, k) = 0.0;
            FLD(s->q3, j, k) = 1.0;
            FLD(s->pr, j, k) = 0.0;
        }
    for (j = 1; j <= s->n2m; j++) {
        s->qb3s[j] = 1.0;
        s->qb3n[j] = 1.0;
    }
    coetar(s);
    if (nlm > 0) {
        memcpy(s->vert, vert, sizeof(double) * 2 * (size_t)(nlm + 1));
        rigid_setup(s);
    }
    return s;
}

void fbo_destroy(fbo_state *s)
{
    if (!s) return;
    void **pp[] = {
        (void **)&s->rc, (void **)&s->rm, (void **)&s->zz, (void **)&s->zm, (void **)&s->g2rc,
        (void **)&s->g2rm, (void **)&s->g3rc, (void **)&s->g3rm, (void **)&s->udx2c,
        (void **)&s->udx2m, (void **)&s->udx3c, (void **)&s->udx3m, (void **)&s->jmv,
        (void **)&s->jpv, (void **)&s->jmc, (void **)&s->jpc, (void **)&s->kmv, (void **)&s->kpv,
        (void **)&s->kmc, (void **)&s->kpc, (void **)&s->am2j, (void **)&s->ac2j,
        (void **)&s->ap2j, (void **)&s->am3j, (void **)&s->ac3j, (void **)&s->ap3j,
        (void **)&s->am3ck, (void **)&s->ac3ck, (void **)&s->ap3ck, (void **)&s->am3sk,
        (void **)&s->ac3sk, (void **)&s->ap3sk, (void **)&s->amphj, (void **)&s->acphj,
        (void **)&s->apphj, (void **)&s->amphk, (void **)&s->acphk, (void **)&s->apphk,
        (void **)&s->wr, (void **)&s->zmm, (void **)&s->zmmt, (void **)&s->q2, (void **)&s->q3,
        (void **)&s->pr, (void **)&s->dph, (void **)&s->q2f, (void **)&s->q3f, (void **)&s->rhs,
        (void **)&s->rhs2, (void **)&s->rhs3, (void **)&s->ru2, (void **)&s->ru3,
        (void **)&s->qcap, (void **)&s->fey, (void **)&s->fez, (void **)&s->hmn,
        (void **)&s->vmn, (void **)&s->qb2s, (void **)&s->qb2n, (void **)&s->dqb2s,
        (void **)&s->dqb2n, (void **)&s->qb3s, (void **)&s->qb3n, (void **)&s->dqb3s,
        (void **)&s->dqb3n, (void **)&s->dq2x2o, (void **)&s->dq3x2o, (void **)&s->lmcc,
        (void **)&s->lmvel, (void **)&s->lmacc, (void **)&s->lmnor, (void **)&s->lmA,
        (void **)&s->vert, (void **)&s->lmind, (void **)&s->eulins, (void **)&s->phi,
        (void **)&s->cl, (void **)&s->press, (void **)&s->tau, (void **)&s->bcerrv,
        (void **)&s->bcerrw, (void **)&s->snap};
    for (size_t i = 0; i < sizeof(pp) / sizeof(pp[0]); i++) free(*pp[i]);
    free(s);
}

void fbo_set_eigen(fbo_state *s, const double *wr, const double *zmm, const double *zmmt)
{
    size_t n = (size_t)s->n3m;
    memcpy(s->wr, wr, n * sizeof(double));
    memcpy(s->zmm, zmm, n * n * sizeof(double));
    memcpy(s->zmmt, zmmt, n * n * sizeof(double));
}

/* ----------------------------------------------------------- fluid stages */

/* cfl.F90:4-51 (here fluid_tsch.F90:211-258) */
static void cfl(fbo_state *s)
{
    int n2 = s->n2, j, k, jp, kp;
    double my_cflm = 1.0e-8, myq3avg = 0.0, qcf, udx3, udx2;
    for (k = 1; k <= s->n3m; k++) {
        udx3 = s->udx3m[k];
        kp = k + 1;
        for (j = 1; j <= s->n2m; j++) {
            udx2 = s->udx2m[j];
            jp = j + 1;
            qcf = (fabs((FLD(s->q2, j, k) + FLD(s->q2, jp, k)) * 0.5 * udx2) +
                   fabs((FLD(s->q3, j, k) + FLD(s->q3, j, kp)) * 0.5 * udx3));
            my_cflm = dmax(my_cflm, qcf);
            myq3avg = myq3avg + FLD(s->q3, j, k) * (s->zz[kp] - s->zz[k]) * (s->rc[jp] - s->rc[j]);
        }
    }
    s->cflm = my_cflm;
    s->q3avg = myq3avg / (s->p.rext2 * s->p.alx3);
}

/* iobcs.F90:5-77 */
static void boucdq(fbo_state *s)
{
    int n2 = s->n2, n3 = s->n3, n3m = s->n3m, j;
    double dq2x2, dq3x2, area, darea, qout, qinf, cor;
    for (j = 1; j <= n2; j++) {
        s->dqb2s[j] = 0.0;
        s->dqb3s[j] = 0.0;
    }
    for (j = 1; j <= s->n2m; j++) {
        dq2x2 = (s->qb2n[j] - FLD(s->q2, j, n3m)) * 2.0 * s->udx3c[n3];
        s->dqb2n[j] = -s->dt * (s->ga * dq2x2 + s->ro * s->dq2x2o[j]) * s->p.cou;
        dq3x2 = (s->qb3n[j] - FLD(s->q3, j, n3m)) * s->udx3c[n3];
        s->dqb3n[j] = -s->dt * (s->ga * dq3x2 + s->ro * s->dq3x2o[j]) * s->p.cou;
        s->dq2x2o[j] = dq2x2;
        s->dq3x2o[j] = dq3x2;
    }
    area = 0.0;
    qout = 0.0;
    qinf = 0.0;
    for (j = 1; j <= s->n2m; j++) {
        darea = s->g2rm[j] / s->dx2;
        area = area + darea;
        qout = qout + s->dqb3n[j] * darea;
        qinf = qinf + s->dqb3s[j] * darea;
    }
    cor = (qinf - qout) / area;
    for (j = 1; j <= s->n2m; j++) s->dqb3n[j] = s->dqb3n[j] + cor;
}

/* iobcs.F90:81-108 */
static void boucqt(fbo_state *s)
{
    int j;
    for (j = 1; j <= s->n2m; j++) {
        s->qb2s[j] = s->qb2s[j] + s->dqb2s[j];
        s->qb3s[j] = s->qb3s[j] + s->dqb3s[j];
        s->qb2n[j] = s->qb2n[j] + s->dqb2n[j];
        s->qb3n[j] = s->qb3n[j] + s->dqb3n[j];
    }
}

/* HDNL.F90:5-110 */
static void hdnl2(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double *q2 = s->q2, *q3 = s->q3;
    double *dph = s->dph;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++) {
        int jc, jm, jp;
        for (jc = 2; jc <= n2m; jc++) {
            double h22;
            jm = jc - 1;
            jp = jc + 1;
            h22 = ((FLD(q2, jp, kc) + FLD(q2, jc, kc)) * (FLD(q2, jp, kc) + FLD(q2, jc, kc)) -
                   (FLD(q2, jm, kc) + FLD(q2, jc, kc)) * (FLD(q2, jm, kc) + FLD(q2, jc, kc))) *
                  s->udx2c[jc] * 0.25;
            FLD(dph, jc, kc) = -h22;
        }
    }
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m - 1; kc++) {
        int kmm = s->kmv[kc], kpp = s->kpv[kc], kp = kc + 1, jc, jm;
        for (jc = 2; jc <= n2m; jc++) {
            double h23;
            jm = s->jmv[jc];
            h23 = ((FLD(q3, jc, kp) + FLD(q3, jm, kp)) * (FLD(q2, jc, kpp) + FLD(q2, jc, kc)) -
                   (FLD(q3, jc, kc) + FLD(q3, jm, kc)) * (FLD(q2, jc, kc) + FLD(q2, jc, kmm))) *
                  s->udx3m[kc] * 0.25;
            FLD(dph, jc, kc) = FLD(dph, jc, kc) - h23;
        }
    }
    {   /* outflow */
        int kc2 = n3m, kmm = kc2 - 1, jc, jm;
        for (jc = 2; jc <= n2m; jc++) {
            double h23;
            jm = s->jmv[jc];
            h23 = (s->qb2n[jc] * (s->qb3n[jc] + s->qb3n[jm]) -
                   (FLD(q3, jc, kc2) + FLD(q3, jm, kc2)) * (FLD(q2, jc, kc2) + FLD(q2, jc, kmm)) * 0.5) *
                  s->udx3m[kc2] * 0.5;
            FLD(dph, jc, kc2) = FLD(dph, jc, kc2) - h23;
        }
    }
    {   /* inflow */
        int kc2 = 1, kp = kc2 + 1, jc, jm;
        for (jc = 2; jc <= n2m; jc++) {
            double h23;
            jm = s->jmv[jc];
            h23 = ((FLD(q3, jc, kp) + FLD(q3, jm, kp)) * (FLD(q2, jc, kc2) + FLD(q2, jc, kp)) * 0.5 -
                   s->qb2s[jc] * (s->qb3s[jc] + s->qb3s[jm])) *
                  s->udx3m[kc2] * 0.5;
            FLD(dph, jc, kc2) = FLD(dph, jc, kc2) - h23;
        }
    }
}

/* HDNL.F90:114-171 */
static void hdnl3(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double *q2 = s->q2, *q3 = s->q3;
    double *qcap = s->qcap;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m - 1; kc++) {
        int kmm = kc - 1, km = s->kmv[kc], kp = kc + 1, jc;
        for (jc = 1; jc <= n2m; jc++) {
            int jmm = s->jmv[jc], jpp = s->jpv[jc], jp = jc + 1;
            double h32, h33;
            h32 = (((FLD(q2, jp, kc) + FLD(q2, jp, km)) * (FLD(q3, jpp, kc) + FLD(q3, jc, kc))) -
                   ((FLD(q2, jc, kc) + FLD(q2, jc, km)) * (FLD(q3, jc, kc) + FLD(q3, jmm, kc)))) *
                  s->udx2m[jc] * 0.25;
            h33 = ((FLD(q3, jc, kp) + FLD(q3, jc, kc)) * (FLD(q3, jc, kp) + FLD(q3, jc, kc)) -
                   (FLD(q3, jc, kc) + FLD(q3, jc, kmm)) * (FLD(q3, jc, kc) + FLD(q3, jc, kmm))) *
                  s->udx3c[kc] * 0.25;
            FLD(qcap, jc, kc) = -(h32 + h33);
        }
    }
}

/* INVTR.F90:4-152 */
static void invtr2(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double al = s->al, ga = s->ga, ro = s->ro, dt = s->dt, alre = al / s->ren;
    double *q2 = s->q2, *pr = s->pr, *rhs2 = s->rhs2, *dph = s->dph, *ru2 = s->ru2, *q2f = s->q2f;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m - 1; kc++) {
        int km = s->kmv[kc], kp = s->kpv[kc], jc;
        double amm = s->am3sk[kc], acc = s->ac3sk[kc], app = s->ap3sk[kc];
        for (jc = 2; jc <= n2m; jc++) {
            int jm = jc - 1, jp = jc + 1;
            double ammj = s->am2j[jc], accj = s->ac2j[jc], appj = s->ap2j[jc];
            double udx2 = al * s->udx2c[jc];
            double d22q2 = FLD(q2, jp, kc) * appj + FLD(q2, jc, kc) * accj + FLD(q2, jm, kc) * ammj;
            double d33q2 = FLD(q2, jc, kp) * app + FLD(q2, jc, kc) * acc + FLD(q2, jc, km) * amm;
            double dcq2 = d22q2 + d33q2;
            double dpx22 = (FLD(pr, jc, kc) - FLD(pr, jm, kc)) * udx2;
            FLD(rhs2, jc, kc) = (ga * FLD(dph, jc, kc) + ro * FLD(ru2, jc, kc) + alre * dcq2 - dpx22) * dt;
            FLD(ru2, jc, kc) = FLD(dph, jc, kc);
        }
    }
    {
        int kc2 = 1, kp = kc2 + 1, jc;
        double codea = s->dx3q / (s->g3rc[kp] * s->g3rm[kc2]);
        double codeb = s->dx3q / (s->g3rc[kc2] * s->g3rm[kc2]);
        for (jc = 2; jc <= n2m; jc++) {
            int jp = jc + 1, jm = jc - 1;
            double ammj = s->am2j[jc], accj = s->ac2j[jc], appj = s->ap2j[jc];
            double d22q2 = FLD(q2, jp, kc2) * appj + FLD(q2, jc, kc2) * accj + FLD(q2, jm, kc2) * ammj;
            double d33q2 = ((FLD(q2, jc, kp) - FLD(q2, jc, kc2)) * codea -
                            (FLD(q2, jc, kc2) - s->qb2s[jc]) * codeb * 2.0);
            double dcq2 = d22q2 + d33q2;
            double dpx22 = (FLD(pr, jc, kc2) - FLD(pr, jm, kc2)) * s->udx2c[jc] * al;
            FLD(rhs2, jc, kc2) = +(ga * FLD(dph, jc, kc2) + ro * FLD(ru2, jc, kc2) + alre * dcq2 - dpx22) * dt;
            FLD(ru2, jc, kc2) = FLD(dph, jc, kc2);
        }
    }
    {
        int kc2 = n3m, km = kc2 - 1, kp = kc2 + 1, jc;
        double codea = s->dx3q / (s->g3rc[kp] * s->g3rm[kc2]);
        double codeb = s->dx3q / (s->g3rc[kc2] * s->g3rm[kc2]);
        for (jc = 2; jc <= n2m; jc++) {
            int jm = jc - 1, jp = jc + 1;
            double ammj = s->am2j[jc], accj = s->ac2j[jc], appj = s->ap2j[jc];
            double d22q2 = FLD(q2, jp, kc2) * appj + FLD(q2, jc, kc2) * accj + FLD(q2, jm, kc2) * ammj;
            double d33q2 = ((s->qb2n[jc] - FLD(q2, jc, kc2)) * codea * 2.0 -
                            (FLD(q2, jc, kc2) - FLD(q2, jc, km)) * codeb);
            double dcq2 = d22q2 + d33q2;
            double dpx22 = (FLD(pr, jc, kc2) - FLD(pr, jm, kc2)) * s->udx2c[jc] * al;
            FLD(rhs2, jc, kc2) = +(ga * FLD(dph, jc, kc2) + ro * FLD(ru2, jc, kc2) + alre * dcq2 - dpx22) * dt;
            FLD(ru2, jc, kc2) = FLD(dph, jc, kc2);
        }
    }
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++) {
        int jc;
        for (jc = 2; jc <= n2m; jc++) FLD(q2f, jc, kc) = FLD(q2, jc, kc) + FLD(rhs2, jc, kc);
    }
}

/* INVTR.F90:156-280 */
static void invtr3(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double al = s->al, ga = s->ga, ro = s->ro, dt = s->dt, alre = al / s->ren;
    const double q3lw = s->p.q3lw, q3uw = s->p.q3uw;
    double *q3 = s->q3, *pr = s->pr, *rhs3 = s->rhs3, *qcap = s->qcap, *ru3 = s->ru3, *q3f = s->q3f;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m; kc++) {
        int km = kc - 1, kp = kc + 1, jc, jm, jp;
        double udx3 = al * s->udx3c[kc];
        double amm = s->am3ck[kc], acc = s->ac3ck[kc], app = s->ap3ck[kc];
        double ammj, accj, appj, dq32, dq33, dcq3, dpx33;
        jc = 1;
        jp = jc + 1;
        ammj = s->am3j[jc]; accj = s->ac3j[jc]; appj = s->ap3j[jc];
        dq32 = FLD(q3, jp, kc) * appj + FLD(q3, jc, kc) * accj + q3lw * ammj;
        dq33 = FLD(q3, jc, kp) * app + FLD(q3, jc, kc) * acc + FLD(q3, jc, km) * amm;
        dcq3 = dq32 + dq33;
        dpx33 = (FLD(pr, jc, kc) - FLD(pr, jc, km)) * udx3;
        FLD(rhs3, jc, kc) = (ga * FLD(qcap, jc, kc) + ro * FLD(ru3, jc, kc) + alre * dcq3 - dpx33) * dt;
        FLD(ru3, jc, kc) = FLD(qcap, jc, kc);
        for (jc = 2; jc <= n2m - 1; jc++) {
            jm = s->jmv[jc];
            jp = s->jpv[jc];
            ammj = s->am3j[jc]; accj = s->ac3j[jc]; appj = s->ap3j[jc];
            dq32 = FLD(q3, jp, kc) * appj + FLD(q3, jc, kc) * accj + FLD(q3, jm, kc) * ammj;
            dq33 = FLD(q3, jc, kp) * app + FLD(q3, jc, kc) * acc + FLD(q3, jc, km) * amm;
            dcq3 = dq32 + dq33;
            dpx33 = (FLD(pr, jc, kc) - FLD(pr, jc, km)) * udx3;
            FLD(rhs3, jc, kc) = (ga * FLD(qcap, jc, kc) + ro * FLD(ru3, jc, kc) + alre * dcq3 - dpx33) * dt;
            FLD(ru3, jc, kc) = FLD(qcap, jc, kc);
        }
        jc = n2m;
        jm = jc - 1;
        ammj = s->am3j[jc]; accj = s->ac3j[jc]; appj = s->ap3j[jc];
        dq32 = q3uw * appj + FLD(q3, jc, kc) * accj + FLD(q3, jm, kc) * ammj;
        dq33 = FLD(q3, jc, kp) * app + FLD(q3, jc, kc) * acc + FLD(q3, jc, km) * amm;
        dcq3 = dq32 + dq33;
        dpx33 = (FLD(pr, jc, kc) - FLD(pr, jc, km)) * udx3;
        FLD(rhs3, jc, kc) = (ga * FLD(qcap, jc, kc) + ro * FLD(ru3, jc, kc) + alre * dcq3 - dpx33) * dt;
        FLD(ru3, jc, kc) = FLD(qcap, jc, kc);
    }
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m; kc++) {
        int jc;
        for (jc = 1; jc <= n2m; jc++) FLD(q3f, jc, kc) = FLD(q3, jc, kc) + FLD(rhs3, jc, kc);
    }
}

/* solve_fluid.F90:110-160 */
static void solq2j(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double betadx = s->beta * s->al;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++) {
        double amjl[n2 + 1], apjl[n2 + 1], acjl[n2 + 1], fjl[n2 + 1], du2[n2 + 1];
        int ipiv[n2 + 1], jc;
        apjl[1] = 0.0; acjl[1] = 1.0; amjl[1] = 0.0;
        apjl[n2] = 0.0; acjl[n2] = 1.0; amjl[n2] = 0.0;
        fjl[1] = 0.0;
        for (jc = 2; jc <= n2m; jc++) {
            double acjl_b = 1.0 / (1.0 - betadx * s->ac2j[jc]);
            apjl[jc] = -betadx * s->ap2j[jc] * acjl_b;
            acjl[jc] = 1.0;
            amjl[jc] = -betadx * s->am2j[jc] * acjl_b;
            fjl[jc] = FLD(s->rhs, jc, kc) * acjl_b;
        }
        fjl[n2] = 0.0;
        tri_solve(n2, amjl + 2, acjl + 1, apjl + 1, fjl + 1, du2, ipiv);
        for (jc = 1; jc <= n2; jc++) FLD(s->rhs, jc, kc) = fjl[jc];
    }
}

/* solve_fluid.F90:164-229 (transposes collapse on one rank) */
static void solq2k(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double betadx = s->beta * s->al;
    const double ugkks = 1.0 / (s->g3rm[1] * s->g3rc[1]) * s->dx3q * 2.0 * betadx;
    const double ugkkn = 1.0 / (s->g3rm[n3m] * s->g3rc[s->n3]) * s->dx3q * 2.0 * betadx;
    int jc;
#pragma omp parallel for schedule(static)
    for (jc = 1; jc <= n2m; jc++) {
        double amkl[n3m + 2], apkl[n3m + 2], ackl[n3m + 2], fkl[n3m + 2], du2[n3m + 2];
        int ipiv[n3m + 2], kc;
        for (kc = 1; kc <= n3m; kc++) {
            double ackl_b = 1.0 / (1.0 - s->ac3sk[kc] * betadx);
            amkl[kc] = -s->am3sk[kc] * betadx * ackl_b;
            ackl[kc] = 1.0;
            apkl[kc] = -s->ap3sk[kc] * betadx * ackl_b;
            fkl[kc] = FLD(s->rhs, jc, kc) * ackl_b;
        }
        fbo_dgttrf(n3m, amkl + 2, ackl + 1, apkl + 1, du2, ipiv);
        fkl[1] = fkl[1] + s->dqb2s[jc] * ugkks;
        fkl[n3m] = fkl[n3m] + s->dqb2n[jc] * ugkkn;
        fbo_dgtts2(n3m, amkl + 2, ackl + 1, apkl + 1, du2, ipiv, fkl + 1);
        for (kc = 1; kc <= n3m; kc++) FLD(s->rhs, jc, kc) = fkl[kc];
    }
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= n3m; kc++)
        for (int j = 1; j <= n2m; j++) FLD(s->q2, j, kc) = FLD(s->q2, j, kc) + FLD(s->rhs, j, kc);
}

/* solve_fluid.F90:61-104 */
static void solq3j(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double betadx = s->beta * s->al;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++) {
        double amjl[n2 + 1], apjl[n2 + 1], acjl[n2 + 1], fjl[n2 + 1], du2[n2 + 1];
        int ipiv[n2 + 1], jc;
        for (jc = 1; jc <= n2m; jc++) {
            double acjl_b = 1.0 / (1.0 - betadx * s->ac3j[jc]);
            apjl[jc] = -betadx * s->ap3j[jc] * acjl_b;
            acjl[jc] = 1.0;
            amjl[jc] = -betadx * s->am3j[jc] * acjl_b;
            fjl[jc] = FLD(s->rhs, jc, kc) * acjl_b;
        }
        tri_solve(n2m, amjl + 2, acjl + 1, apjl + 1, fjl + 1, du2, ipiv);
        for (jc = 1; jc <= n2m; jc++) FLD(s->rhs, jc, kc) = fjl[jc];
    }
}

/* solve_fluid.F90:233-312 */
static void solq3k(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m, n3 = s->n3;
    const double betadx = s->beta * s->al;
    int jc;
#pragma omp parallel for schedule(static)
    for (jc = 1; jc <= n2m; jc++) {
        double amkl[n3 + 2], apkl[n3 + 2], ackl[n3 + 2], fkl[n3 + 2], du2[n3 + 2];
        int ipiv[n3 + 2], kc;
        amkl[1] = 0.0; apkl[1] = 0.0; ackl[1] = 1.0;
        amkl[n3] = 0.0; apkl[n3] = 0.0; ackl[n3] = 1.0;
        fkl[1] = s->dqb3s[jc];
        for (kc = 2; kc <= n3m; kc++) {
            double ackl_b = 1.0 / (1.0 - s->ac3sk[kc] * betadx);
            amkl[kc] = -s->am3sk[kc] * betadx * ackl_b;
            ackl[kc] = 1.0;
            apkl[kc] = -s->ap3sk[kc] * betadx * ackl_b;
            fkl[kc] = FLD(s->rhs, jc, kc) * ackl_b;
        }
        fkl[n3] = s->dqb3n[jc];
        tri_solve(n3, amkl + 2, ackl + 1, apkl + 1, fkl + 1, du2, ipiv);
        for (kc = 1; kc <= n3m; kc++) FLD(s->rhs, jc, kc) = fkl[kc];
    }
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= n3m; kc++)
        for (int j = 1; j <= n2m; j++) FLD(s->q3, j, kc) = FLD(s->q3, j, kc) + FLD(s->rhs, j, kc);
    for (jc = 1; jc <= n2m; jc++) FLD(s->q3, jc, n3) = FLD(s->q3, jc, n3) + s->dqb3n[jc];
}

/* helsolve.F90:4-56 */
static void helsolve(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double dt = s->dt;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++)
        for (int jc = 2; jc <= n2m; jc++)
            FLD(s->rhs, jc, kc) = FLD(s->rhs2, jc, kc) + FLD(s->fey, jc, kc) * dt;
    solq2j(s);
    solq2k(s);
    for (kc = -KG; kc <= s->n3 + KG; kc++) {
        FLD(s->q2, n2, kc) = 0.0;
        FLD(s->q2, 1, kc) = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m; kc++)
        for (int jc = 1; jc <= n2m; jc++)
            FLD(s->rhs, jc, kc) = FLD(s->rhs3, jc, kc) + FLD(s->fez, jc, kc) * dt;
    solq3j(s);
    solq3k(s);
}

/* divergence.F90:88-115 */
static void divg(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double usdtal = 1.0 / (s->dt * s->al);
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++) {
        int kp = kc + 1;
        for (int jc = 1; jc <= n2m; jc++) {
            int jp = jc + 1;
            double dqcap = (FLD(s->q2, jp, kc) - FLD(s->q2, jc, kc)) * s->udx2m[jc] +
                           (FLD(s->q3, jc, kp) - FLD(s->q3, jc, kc)) * s->udx3m[kc];
            FLD(s->dph, jc, kc) = dqcap * usdtal;
        }
    }
}

/* phcalc_outflow.F90:4-71; the DGEMMs are summed in netlib order (over the
 * inner index from 1 upward, starting from zero) */
static void phcalc(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    double *hmn = s->hmn, *vmn = s->vmn;
    int k;
    /* hmn(j,k) = sum_m dph(j,m) * zmmt(k,m)   (DGEMM 'n','t') */
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3m; k++) {
        double *c = hmn + (size_t)(k - 1) * n2m;
        for (int j = 0; j < n2m; j++) c[j] = 0.0;
        for (int m = 1; m <= n3m; m++) {
            double t = s->zmmt[(size_t)(k - 1) + (size_t)(m - 1) * n3m];
            const double *a = &FLD(s->dph, 1, m);
            for (int j = 0; j < n2m; j++) c[j] = c[j] + t * a[j];
        }
    }
    /* per-mode tridiagonal in y; vmn stored (j, k) -- the reference's vmn(k,j) */
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3m; k++) {
        double amph[n2m + 2], apph[n2m + 2], acphT[n2m + 2], fphj[n2m + 2], du2[n2m + 2];
        int ipiv[n2m + 2];
        for (int j = 1; j <= n2m; j++) {
            double acphT_b = 1.0 / (s->acphj[j] + s->wr[k - 1]);
            acphT[j] = 1.0;
            apph[j] = s->apphj[j] * acphT_b;
            amph[j] = s->amphj[j] * acphT_b;
            fphj[j] = hmn[(size_t)(k - 1) * n2m + (j - 1)] * acphT_b;
        }
        tri_solve(n2m, amph + 2, acphT + 1, apph + 1, fphj + 1, du2, ipiv);
        for (int j = 1; j <= n2m; j++) vmn[(size_t)(k - 1) * n2m + (j - 1)] = fphj[j];
    }
    /* hmnt(k,j) = sum_m zmm(k,m) vmn(m,j) (DGEMM 'n','n'); dph(j,k) = hmnt(k,j) */
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3m; k++) {
        double *c = &FLD(s->dph, 1, k);
        for (int j = 0; j < n2m; j++) c[j] = 0.0;
        for (int m = 1; m <= n3m; m++) {
            double t = s->zmm[(size_t)(k - 1) + (size_t)(m - 1) * n3m];
            const double *b = vmn + (size_t)(m - 1) * n2m;
            for (int j = 0; j < n2m; j++) c[j] = c[j] + b[j] * t;
        }
    }
}

/* updvp.F90:5-59 */
static void updvp(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double al = s->al, dt = s->dt;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++)
        for (int jc = 1; jc <= n2m; jc++) {
            int jm = s->jmv[jc];
            double usujm = al * dt * s->udx2c[jc];
            double locdph = FLD(s->dph, jc, kc);
            FLD(s->q2, jc, kc) = FLD(s->q2, jc, kc) - (locdph - FLD(s->dph, jm, kc)) * usujm;
        }
#pragma omp parallel for schedule(static)
    for (kc = 2; kc <= n3m; kc++) {
        int km = kc - 1;
        double usukm = al * dt * s->udx3c[kc];
        for (int jc = 1; jc <= n2m; jc++)
            FLD(s->q3, jc, kc) = FLD(s->q3, jc, kc) - (FLD(s->dph, jc, kc) - FLD(s->dph, jc, km)) * usukm;
    }
}

/* updvp.F90:68-105 */
static void prcalc(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    const double be = s->al * s->beta;
    int kc;
#pragma omp parallel for schedule(static)
    for (kc = 1; kc <= n3m; kc++) {
        int kp = s->kpv[kc], km = s->kmv[kc];
        double ammk = s->amphk[kc], acck = s->acphk[kc], appk = s->apphk[kc];
        for (int jc = 1; jc <= n2m; jc++) {
            int jm = s->jmv[jc], jp = s->jpv[jc];
            double ammj = s->amphj[jc], accj = s->acphj[jc], appj = s->apphj[jc];
            FLD(s->pr, jc, kc) =
                FLD(s->pr, jc, kc) + FLD(s->dph, jc, kc) -
                be * ((FLD(s->dph, jp, kc) * appj + FLD(s->dph, jc, kc) * accj + FLD(s->dph, jm, kc) * ammj) +
                      (FLD(s->dph, jc, kp) * appk + FLD(s->dph, jc, kc) * acck + FLD(s->dph, jc, km) * ammk));
        }
    }
}

/* updvp.F90:112-144 */
static void pr_submean(fbo_state *s)
{
    const int n2 = s->n2, n2m = s->n2m, n3m = s->n3m;
    double mypravg = 0.0, pravg;
    size_t i, nf = (size_t)n2 * (size_t)(s->n3 + 1 + 2 * KG);
    for (int k = 1; k <= n3m; k++) {
        int kp = k + 1;
        for (int j = 1; j <= n2m; j++) {
            int jp = j + 1;
            mypravg = mypravg + FLD(s->pr, j, k) * (s->zz[kp] - s->zz[k]) * (s->rc[jp] - s->rc[j]);
        }
    }
    pravg = mypravg / (s->p.rext2 * s->p.alx3);
    s->pravg = pravg;
    for (i = 0; i < nf; i++) s->pr[i] = s->pr[i] - pravg;
}

/* ------------------------------------------------------------ MLS forcing */

/* minloc(abs(a(lo:hi) - x)): first index of the minimum, 1-based in a */
static int minloc_abs(const double *a, int lo, int hi, double x)
{
    int i, best = lo;
    double bv = fabs(a[lo] - x);
    for (i = lo + 1; i <= hi; i++) {
        double v = fabs(a[i] - x);
        if (v < bv) {
            bv = v;
            best = i;
        }
    }
    return best;
}

/* lgrdistribution.F90:189-267 */
static int lgrdistribution(fbo_state *s)
{
    int i, nlm = s->nlm, n2 = s->n2, n3 = s->n3, n2m = s->n2m, n3m = s->n3m;
    double ymax = -1e300, ymin = 1e300, zmax = -1e300, zmin = 1e300;
    for (i = 1; i <= nlm; i++) {
        ymax = fmax(ymax, M2(s->lmcc, i, 1));
        ymin = fmin(ymin, M2(s->lmcc, i, 1));
        zmax = fmax(zmax, M2(s->lmcc, i, 2));
        zmin = fmin(zmin, M2(s->lmcc, i, 2));
    }
    if (ymax > s->p.rext2 || ymin < 0.0 || zmax > s->p.alx3 || zmin < 0.0) return FBO_ERR_MARKER_OUT;
    for (i = 1; i <= nlm; i++) {
        double y = M2(s->lmcc, i, 1), z = M2(s->lmcc, i, 2);
        int ind;
        LMIND(i, 1, 1) = minloc_abs(s->rc, 1, n2, y);
        if (z < s->zm[1] && z > 0.0) ind = 1;
        else if (z > s->zm[n3m] && z < s->p.alx3) ind = n3m;
        else ind = minloc_abs(s->zm, 1, n3, z);
        LMIND(i, 1, 2) = ind;
        if (y < s->rm[1] && y > 0.0) ind = 1;
        else if (y > s->rm[n2m] && y < s->p.rext2) ind = n2m;
        else ind = minloc_abs(s->rm, 1, n2, y);
        LMIND(i, 2, 1) = ind;
        LMIND(i, 2, 2) = minloc_abs(s->zz, 1, n3, z);
    }
    return FBO_OK;
}

/* MLSint.F90:4-104.  Returns nonzero when a support node has no right
 * neighbour on its axis (the reference reads past its copy of the axis
 * there; such a marker is treated as outside the domain). */
static int mls_sd_ind(fbo_state *s, int idir, const int indse[2], double posk[2][9],
                      double dsk[2][9], int eul[2][9])
{
    const double *y, *z;
    int dimy, dimz, j, k, m, e[3][3][2];
    if (idir == 1) {
        y = s->rc; dimy = s->n2; z = s->zm; dimz = s->n3m;
    } else if (idir == 2) {
        y = s->rm; dimy = s->n2m; z = s->zz; dimz = s->n3;
    } else {
        y = s->rm; dimy = s->n2m; z = s->zm; dimz = s->n3m;
    }
    for (j = 1; j <= 3; j++)
        for (k = 1; k <= 3; k++) {
            int jj, kk;
            if (indse[0] == 1) jj = j + 1;
            else if (indse[0] == s->n2m) jj = j - 1;
            else jj = j;
            if (indse[1] == 1) kk = k + 1;
            else if (indse[1] == s->n3m) kk = k - 1;
            else kk = k;
            e[j - 1][k - 1][0] = indse[0] + jj - 2;
            e[j - 1][k - 1][1] = indse[1] + kk - 2;
        }
    m = 0;
    for (j = 1; j <= 3; j++)
        for (k = 1; k <= 3; k++) {
            int ind;
            ind = e[j - 1][k - 1][0];
            if (ind < 1 || ind + 1 > dimy) return 1;
            posk[0][m] = y[ind];
            dsk[0][m] = y[ind + 1] - y[ind];
            ind = e[j - 1][k - 1][1];
            if (ind < 1 || ind + 1 > dimz) return 1;
            posk[1][m] = z[ind];
            dsk[1][m] = z[ind + 1] - z[ind];
            eul[0][m] = e[j - 1][k - 1][0];
            eul[1][m] = e[j - 1][k - 1][1];
            m++;
        }
    return 0;
}

/* utils_math.f90:637-725: Gaussian elimination with scaled partial pivoting.
 * a is (row, col); returns 1 on success, 0 for a singular matrix. */
static int gesolve3(const double ai[3][3], const double bi[3], double x[3])
{
    const int n = 3;
    double a[3][3], b[3], sc[3], c, pivot, store;
    int i, j, k, l;
    memcpy(a, ai, sizeof(a));
    memcpy(b, bi, sizeof(b));
    for (k = 0; k < n - 1; k++) {
        for (i = k; i < n; i++) {
            sc[i] = 0.0;
            for (j = k; j < n; j++) sc[i] = dmax(sc[i], fabs(a[i][j]));
        }
        pivot = fabs(a[k][k] / sc[k]);
        l = k;
        for (j = k + 1; j < n; j++) {
            if (fabs(a[j][k] / sc[j]) > pivot) {
                pivot = fabs(a[j][k] / sc[j]);
                l = j;
            }
        }
        if (pivot == 0.0) return 0;
        if (l != k) {
            for (j = k; j < n; j++) {
                store = a[k][j];
                a[k][j] = a[l][j];
                a[l][j] = store;
            }
            store = b[k];
            b[k] = b[l];
            b[l] = store;
        }
        for (i = k + 1; i < n; i++) {
            c = a[i][k] / a[k][k];
            a[i][k] = 0.0;
            b[i] = b[i] - c * b[k];
            for (j = k + 1; j < n; j++) a[i][j] = a[i][j] - c * a[k][j];
        }
    }
    x[n - 1] = b[n - 1] / a[n - 1][n - 1];
    for (i = n - 2; i >= 0; i--) {
        c = 0.0;
        for (j = i + 1; j < n; j++) c = c + a[i][j] * x[j];
        x[i] = (b[i] - c) / a[i][i];
    }
    return 1;
}

/* cubic-spline and alternative kernels, MLSint.F90:406-486 (one axis) */
static double wkernel(int wfun, double rc)
{
    double rc2 = rc * rc, rc3 = rc * rc * rc, rc4 = rc * rc * rc * rc;
    if (wfun == 1) {
        if (rc > 1.0) return 0.0;
        if (rc <= 0.5) return (2.0 / 3.0) - 4.0 * rc2 + 4.0 * rc3;
        return (4.0 / 3.0) - 4.0 * rc + 4.0 * rc2 - (4.0 / 3.0) * rc3;
    } else if (wfun == 2) {
        if (rc <= 1.0) return exp(-((rc / 0.3) * (rc / 0.3)));
        return 0.0;
    } else if (wfun == 3) {
        if (rc <= 1.0) return 1.0 - 6.0 * rc2 + 8.0 * rc3 - 3.0 * rc4;
        return 0.0;
    } else if (wfun == 4) {
        if (rc > 1.0) return 0.0;
        if (rc < 0.5) return 1.0 / 3.0 * (1.0 + sqrt(-3.0 * rc2 + 1.0));
        return 1.0 / 6.0 * (5.0 - 3.0 * rc - sqrt(-3.0 * ((1.0 - rc) * (1.0 - rc)) + 1.0));
    }
    return 0.0;
}

/* MLSint.F90:115-166 with compute_AB :284-338; returns FBO_ERR_MLS on a
 * partition-of-unity failure */
static int mls_sf(fbo_state *s, const double pos[2], double sdc[2][9], double sdd[2][9],
                  double philoc[9])
{
    double A[3][3], B[3][9], w[9], gps[3], ptA[3], sumphi, errsum;
    int i, j, k;
    for (i = 0; i < 9; i++) {
        double wc[2];
        for (k = 0; k < 2; k++) {
            double difc = pos[k] - sdc[k][i];
            double sdds = s->p.radiusSD * sdd[k][i];
            double rc = fabs(difc) / sdds;
            wc[k] = wkernel(s->p.wfun, rc);
        }
        w[i] = wc[0] * wc[1];
    }
    for (j = 0; j < 9; j++) {
        B[0][j] = 1.0 * w[j];
        B[1][j] = sdc[0][j] * w[j];
        B[2][j] = sdc[1][j] * w[j];
    }
    memset(A, 0, sizeof(A));
    for (i = 0; i < 9; i++) {
        double pk[3] = {1.0, sdc[0][i], sdc[1][i]};
        for (j = 0; j < 3; j++)
            for (k = 0; k < 3; k++) A[j][k] = A[j][k] + w[i] * (pk[j] * pk[k]);
    }
    gps[0] = 1.0;
    gps[1] = pos[0];
    gps[2] = pos[1];
    gesolve3(A, gps, ptA);
    for (j = 0; j < 9; j++) {
        double acc = 0.0;
        for (i = 0; i < 3; i++) acc = acc + ptA[i] * B[i][j];
        philoc[j] = acc;
    }
    sumphi = 0.0;
    for (j = 0; j < 9; j++) sumphi = sumphi + philoc[j];
    errsum = fabs(1.0 - fabs(sumphi));
    if (!(errsum <= 1.0e-10)) return FBO_ERR_MLS;
    return FBO_OK;
}

/* forcing_MLS.F90:5-128 and interp_spread :135-182 */
static int forcing_mls(fbo_state *s, int substep)
{
    const int n2 = s->n2, nlm = s->nlm;
    size_t nf = (size_t)n2 * (size_t)(s->n3 + 1 + 2 * KG);
    int fs, n, st = FBO_OK;
    for (fs = 1; fs <= s->p.forst; fs++) {
        memset(s->fey, 0, nf * sizeof(double));
        memset(s->fez, 0, nf * sizeof(double));
        if (substep == 1 && fs == 1) {
            memset(s->cl, 0, sizeof(double) * 2 * (size_t)nlm);
            memset(s->phi, 0, sizeof(double) * 18 * (size_t)nlm);
        }
        for (n = 1; n <= nlm; n++) {
            double pos[2] = {M2(s->lmcc, n, 1), M2(s->lmcc, n, 2)};
            double areal = s->lmA[n - 1];
            if (!(s->zz[1] < pos[1] && pos[1] < s->zz[s->n3])) continue;
            if (substep == 1 && fs == 1) {
                for (int idir = 1; idir <= 2; idir++) {
                    int indse[2] = {LMIND(n, idir, 1), LMIND(n, idir, 2)};
                    double sdc[2][9], sdd[2][9], ph[9], dvel = 0.0, lgr_h = 0.0;
                    int eul[2][9];
                    if (mls_sd_ind(s, idir, indse, sdc, sdd, eul)) return FBO_ERR_MARKER_OUT;
                    if (mls_sf(s, pos, sdc, sdd, ph) != FBO_OK) st = FBO_ERR_MLS;
                    for (int i = 0; i < 9; i++) {
                        double vol = sdd[0][i] * sdd[1][i];
                        PHI(n, idir, i + 1) = ph[i];
                        dvel = dvel + ph[i] * vol;
                        lgr_h = lgr_h + 1.0 / 2.0 * ph[i] * (sdd[0][i] + sdd[1][i]);
                    }
                    CL(n, idir) = areal * lgr_h / dvel;
                    for (int i = 0; i < 9; i++) {
                        EULINS(n, idir, 1, i + 1) = eul[0][i];
                        EULINS(n, idir, 2, i + 1) = eul[1][i];
                    }
                }
            }
            /* interp_spread */
            {
                double ucy = 0.0, fcy, ucz = 0.0, fcz;
                int i;
                for (i = 1; i <= 9; i++)
                    ucy = ucy + PHI(n, 1, i) * FLD(s->q2f, EULINS(n, 1, 1, i), EULINS(n, 1, 2, i));
                fcy = (M2(s->lmvel, n, 1) - ucy) / s->dt;
                for (i = 1; i <= 9; i++) {
                    int jj = EULINS(n, 1, 1, i), kk = EULINS(n, 1, 2, i);
                    FLD(s->fey, jj, kk) = FLD(s->fey, jj, kk) + CL(n, 1) * PHI(n, 1, i) * fcy;
                }
                for (i = 1; i <= 9; i++)
                    ucz = ucz + PHI(n, 2, i) * FLD(s->q3f, EULINS(n, 2, 1, i), EULINS(n, 2, 2, i));
                fcz = (M2(s->lmvel, n, 2) - ucz) / s->dt;
                for (i = 1; i <= 9; i++) {
                    int jj = EULINS(n, 2, 1, i), kk = EULINS(n, 2, 2, i);
                    FLD(s->fez, jj, kk) = FLD(s->fez, jj, kk) + CL(n, 2) * PHI(n, 2, i) * fcz;
                }
            }
        }
    }
    return st;
}

/* ckbcs.F90:5-86 (phipred equals phi: the all-reduce is over one rank) */
static void checkbcs(fbo_state *s)
{
    const int n2 = s->n2;
    int np;
    double sv = 0.0, sw = 0.0;
    for (np = 1; np <= s->nlm; np++) {
        double pos2 = M2(s->lmcc, np, 2), ucy = 0.0, ucz = 0.0;
        s->bcerrv[np - 1] = 0.0;
        s->bcerrw[np - 1] = 0.0;
        if (!(s->zz[1] < pos2 && pos2 < s->zz[s->n3])) continue;
        for (int n = 1; n <= 9; n++)
            ucy = ucy + PHI(np, 1, n) * FLD(s->q2, EULINS(np, 1, 1, n), EULINS(np, 1, 2, n));
        s->bcerrv[np - 1] = M2(s->lmvel, np, 1) - ucy;
        for (int n = 1; n <= 9; n++)
            ucz = ucz + PHI(np, 2, n) * FLD(s->q3, EULINS(np, 2, 1, n), EULINS(np, 2, 2, n));
        s->bcerrw[np - 1] = M2(s->lmvel, np, 2) - ucz;
    }
    for (np = 0; np < s->nlm; np++) {
        sv = sv + s->bcerrv[np] * s->bcerrv[np];
        sw = sw + s->bcerrw[np] * s->bcerrw[np];
    }
    s->nbcv = sqrt(sv) / (double)s->nlm;
    s->nbcw = sqrt(sw) / (double)s->nlm;
}

/* -------------------------------------------------------------- loads */

/* loads_transfer.F90:238-281 */
static int probeind(fbo_state *s, const int markind[2], const double probepos[2], int idir, int ind[2])
{
    const int off = 5;
    int js = markind[0] - off, je = markind[0] + off, ks = markind[1] - off, ke = markind[1] + off;
    const double *ya, *za;
    if (idir == 1) ya = s->rc, za = s->zm;
    else if (idir == 2) ya = s->rm, za = s->zz;
    else ya = s->rm, za = s->zm;
    if (js < 1 || je > s->n2 || ks < 1 || ke > s->n3) return 1;
    ind[0] = minloc_abs(ya, js, je, probepos[0]);
    ind[1] = minloc_abs(za, ks, ke, probepos[1]);
    return 0;
}

/* MLSint.F90:173-258 with compute_AB_d :342-402, weight_function_d :492-593 */
static int mls_sf_d(fbo_state *s, const double pos[2], double sdc[2][9], double sdd[2][9],
                    double phid[3][9])
{
    double w[9][3], A[3][3][3], B[3][9][3], gam[3][3], C[3], gp[3][3], Aa[3][3];
    int i, j, k, l;
    const int wfun = s->p.wfun;
    for (i = 0; i < 9; i++) {
        double wc[2] = {0.0, 0.0}, dw[2] = {0.0, 0.0};
        for (k = 0; k < 2; k++) {
            double difc = pos[k] - sdc[k][i];
            double sdds = s->p.radiusSD * sdd[k][i];
            double drdc, rc, rc2, rc3, rc4;
            if (fabs(difc) <= 1.0e-20) drdc = 0.0;
            else drdc = (difc / fabs(difc)) / sdds;
            rc = fabs(difc) / sdds;
            rc2 = rc * rc;
            rc3 = rc * rc * rc;
            rc4 = rc * rc * rc * rc;
            if (wfun == 1) {
                if (rc > 1.0) {
                    wc[k] = 0.0;
                    dw[k] = 0.0;
                } else if (rc <= 0.5) {
                    wc[k] = (2.0 / 3.0) - 4.0 * rc2 + 4.0 * rc3;
                    dw[k] = (-8.0 * rc + 12.0 * rc2) * drdc;
                } else {
                    wc[k] = (4.0 / 3.0) - 4.0 * rc + 4.0 * rc2 - (4.0 / 3.0) * rc3;
                    dw[k] = (-4.0 + 8.0 * rc - 4.0 * rc2) * drdc;
                }
            } else if (wfun == 2) {
                if (rc <= 1.0) {
                    wc[k] = exp(-((rc / 0.3) * (rc / 0.3)));
                    dw[k] = (-1.0 / (0.3 * 0.3) * 2.0 * rc * exp(-((rc / 0.3) * (rc / 0.3)))) * drdc;
                }
            } else if (wfun == 3) {
                if (rc <= 1.0) {
                    wc[k] = 1.0 - 6.0 * rc2 + 8.0 * rc3 - 3.0 * rc4;
                    dw[k] = -12.0 * rc + 24.0 * rc2 - 12.0 * rc3;
                }
            } else if (wfun == 4) {
                if (rc > 1.0) {
                } else if (rc < 0.5) {
                    wc[k] = 1.0 / 3.0 * (1.0 + sqrt(-3.0 * rc2 + 1.0));
                    dw[k] = -rc * pow(-3.0 * rc2 - 1.0, -0.5);
                } else {
                    wc[k] = 1.0 / 6.0 * (5.0 - 3.0 * rc - sqrt(-3.0 * ((1.0 - rc) * (1.0 - rc)) + 1.0));
                    dw[k] = -(1.0 - rc) / (2.0 * sqrt(1.0 - 3.0 * ((1.0 - rc) * (1.0 - rc)))) - 0.5;
                }
            }
        }
        w[i][0] = wc[0] * wc[1];
        w[i][1] = wc[1] * dw[0];
        w[i][2] = wc[0] * dw[1];
    }
    for (i = 0; i < 9; i++) {
        double pk[3] = {1.0, sdc[0][i], sdc[1][i]};
        for (j = 0; j < 3; j++)
            for (k = 0; k < 3; k++) B[j][i][k] = pk[j] * w[i][k];
    }
    memset(A, 0, sizeof(A));
    for (i = 0; i < 9; i++) {
        double pk[3] = {1.0, sdc[0][i], sdc[1][i]}, pp[3][3];
        for (j = 0; j < 3; j++)
            for (k = 0; k < 3; k++) pp[j][k] = pk[j] * pk[k];
        for (j = 0; j < 3; j++)
            for (k = 0; k < 3; k++)
                for (l = 0; l < 3; l++) A[j][k][l] = A[j][k][l] + w[i][l] * pp[j][k];
    }
    memset(gp, 0, sizeof(gp));
    gp[0][0] = gp[1][1] = gp[2][2] = 1.0;
    gp[0][1] = pos[0];
    gp[0][2] = pos[1];
    for (j = 0; j < 3; j++)
        for (k = 0; k < 3; k++) Aa[j][k] = A[j][k][0];
    {
        double g0[3], gx[3];
        int ok = gesolve3(Aa, gp[0], g0);
        for (l = 1; l <= 2; l++) {
            for (j = 0; j < 3; j++) {
                double acc = 0.0;
                for (k = 0; k < 3; k++) acc = acc + A[j][k][l] * g0[k];
                C[j] = gp[l][j] - acc;
            }
            ok &= gesolve3(Aa, C, gx);
            for (j = 0; j < 3; j++) gam[j][l] = gx[j];
        }
        for (j = 0; j < 3; j++) gam[j][0] = g0[j];
        (void)ok;
    }
    for (i = 0; i < 9; i++) {
        phid[0][i] = phid[1][i] = phid[2][i] = 0.0;
        for (j = 0; j < 3; j++) {
            phid[0][i] = phid[0][i] + gam[j][0] * B[j][i][0];
            phid[1][i] = phid[1][i] + gam[j][1] * B[j][i][0] + gam[j][0] * B[j][i][1];
            phid[2][i] = phid[2][i] + gam[j][2] * B[j][i][0] + gam[j][0] * B[j][i][2];
        }
    }
    {
        double sumphi = 0.0, errsum;
        for (i = 0; i < 9; i++) sumphi = sumphi + phid[0][i];
        errsum = fabs(1.0 - fabs(sumphi));
        if (!(errsum <= 1.0e-10)) return FBO_ERR_MLS;
    }
    return FBO_OK;
}

/* loads_transfer.F90:285-357 (getpbup) for one interpolated quantity */
static void getpbup_one(fbo_state *s, const double *f, const int eul[2][9], const double ph[3][9],
                        double out[7])
{
    const int n2 = s->n2;
    int n, i;
    for (i = 0; i < 7; i++) out[i] = 0.0;
    for (n = 0; n < 9; n++) {
        int cyk = eul[0][n], czk = eul[1][n];
        double uk[3];
        uk[0] = FLD(f, cyk, czk);
        uk[1] = (FLD(f, cyk, czk) - FLD(f, cyk - 1, czk)) * s->dx2 / s->g2rc[cyk];
        uk[2] = (FLD(f, cyk, czk) - FLD(f, cyk, czk - 1)) * s->dx3 / s->g3rc[czk];
        for (i = 0; i < 3; i++) out[i] = out[i] + ph[i][n] * uk[0];
        for (i = 0; i < 2; i++) out[i + 3] = out[i + 3] + ph[1][n] * uk[1 + i];
        for (i = 0; i < 2; i++) out[i + 5] = out[i + 5] + ph[2][n] * uk[1 + i];
    }
}

/* loads_transfer.F90:93-234 (loads_transfer_c) */
static int loads_transfer(fbo_state *s)
{
    const double hpr = s->ddmin * s->p.kprobe, visc = s->p.visc;
    double lmtan[2] = {0.0, 0.0};
    int n, st = FBO_OK;
    for (n = 0; n < s->nlm; n++) {
        s->press[n] = 0.0;
        s->tau[2 * n] = s->tau[2 * n + 1] = 0.0;
    }
    for (n = 1; n <= s->nlm; n++) {
        double pos[2] = {M2(s->lmcc, n, 1), M2(s->lmcc, n, 2)};
        double probe[2] = {pos[0] + M2(s->lmnor, n, 1) * hpr, pos[1] + M2(s->lmnor, n, 2) * hpr};
        double phL[3][3][9], ucy[7], ucz[7], pc[7];
        int eulL[3][2][9];
        if (!(s->zz[1] < pos[1] && pos[1] < s->zz[s->n3])) continue;
        for (int idir = 1; idir <= 3; idir++) {
            int tmp[2], indse[2];
            double sdc[2][9], sdd[2][9];
            if (idir == 3) {
                tmp[0] = LMIND(n, 2, 1);
                tmp[1] = LMIND(n, 1, 2);
            } else {
                tmp[0] = LMIND(n, idir, 1);
                tmp[1] = LMIND(n, idir, 2);
            }
            if (probeind(s, tmp, probe, idir, indse)) return FBO_ERR_MARKER_OUT;
            if (mls_sd_ind(s, idir, indse, sdc, sdd, eulL[idir - 1])) return FBO_ERR_MARKER_OUT;
            if (eulL[idir - 1][0][0] < 2) return FBO_ERR_MARKER_OUT; /* j-1 would leave the array */
            if (mls_sf_d(s, probe, sdc, sdd, phL[idir - 1]) != FBO_OK) st = FBO_ERR_MLS;
        }
        getpbup_one(s, s->q2, eulL[0], phL[0], ucy);
        getpbup_one(s, s->q3, eulL[1], phL[1], ucz);
        getpbup_one(s, s->pr, eulL[2], phL[2], pc);
        {
            double nory = M2(s->lmnor, n, 1), norz = M2(s->lmnor, n, 2);
            double vel[2] = {ucy[0], ucz[0]}, veln_md, veln[2], velt[2], velt_md;
            double tany, tanz, dpdnw, dpdne, ducdn, d3ucdn3, d2ucdn2, ducdnm;
            veln_md = vel[0] * nory + vel[1] * norz;
            veln[0] = veln_md * nory;
            veln[1] = veln_md * norz;
            velt[0] = vel[0] - veln[0];
            velt[1] = vel[1] - veln[1];
            velt_md = sqrt(velt[0] * velt[0] + velt[1] * velt[1]);
            if (velt_md != 0.0) {
                lmtan[0] = velt[0] / sqrt(velt[0] * velt[0] + velt[1] * velt[1]);
                lmtan[1] = velt[1] / sqrt(velt[0] * velt[0] + velt[1] * velt[1]);
            }
            tany = lmtan[0];
            tanz = lmtan[1];
            dpdnw = M2(s->lmacc, n, 1) * nory + M2(s->lmacc, n, 2) * norz;
            dpdnw = -1.0 * dpdnw;
            dpdne = pc[1] * nory + pc[2] * norz;
            s->press[n - 1] = pc[0] - 0.5 * (dpdnw + dpdne) * hpr;
            ducdn = (ucy[1] * tany * nory + ucy[2] * tany * norz + ucz[1] * tanz * nory +
                     ucz[2] * tanz * norz);
            d3ucdn3 = (pc[3] * nory * nory + pc[4] * nory * norz + pc[5] * norz * nory +
                       pc[6] * norz * norz) * 1.0 / visc;
            d2ucdn2 = (ucy[3] * tany * nory * nory + ucy[4] * tany * nory * norz +
                       ucy[5] * tany * norz * nory + ucy[6] * tany * norz * norz +
                       ucz[3] * tanz * nory * nory + ucz[4] * tanz * nory * norz +
                       ucz[5] * tanz * norz * nory + ucz[6] * tanz * norz * norz);
            ducdnm = ducdn - d2ucdn2 * hpr - 0.5 * d3ucdn3 * (hpr * hpr);
            s->tau[2 * (n - 1)] = visc * ducdnm * lmtan[0];
            s->tau[2 * (n - 1) + 1] = visc * ducdnm * lmtan[1];
        }
    }
    return st;
}

/* -------------------------------------------------------------- rigid */

/* rigid.F90:341-369 */
static void modfn(double K[6], const double t[6], const double FF[6], const double Mi[3],
                  const double c[3], const double k1[3], const double k3[3])
{
    for (int i = 0; i < 3; i++) {
        double cube = t[i] * t[i] * t[i];
        double lin = -k1[i] * t[i] + -c[i] * t[i + 3];
        double rhs = lin + -k3[i] * cube + FF[i + 3];
        K[i] = t[i + 3];
        K[i + 3] = Mi[i] * rhs;
    }
}

/* rigid.F90:165-228 (kinem_RK4) and :233-299 (kinem_RK4i) */
static void kinem(fbo_state *s, double Fy, double Fz, double M)
{
    const double dt = s->dt, rhom = s->p.rbden, rr = s->p.rrr;
    double xo[6], xn[6], K1[6], K2[6], K3[6], K4[6], t1[6], t2[6], t3[6], FF[6], Mi[3];
    int i;
    for (i = 0; i < 3; i++) xo[i] = CMP_N[i] - (i < 2 ? s->p.cmposi[i] : s->p.cmroti);
    for (i = 0; i < 3; i++) xo[i + 3] = CMV_N[i];
    FF[0] = FF[1] = FF[2] = 0.0;
    FF[4] = Fz;
    FF[5] = M;
    if (s->p.rtcoup) {
        FF[3] = Fy + M / rr;
        Mi[0] = 1.0 / ((s->p.rba[1] / (rr * rr) + s->p.rba[0]) * rhom);
    } else {
        FF[3] = Fy;
        Mi[0] = 1.0 / (s->p.rba[0] * rhom);
    }
    Mi[1] = 1.0 / (s->p.rba[0] * rhom);
    Mi[2] = 1.0 / (s->p.rba[1] * rhom);
    modfn(K1, xo, FF, Mi, s->p.cc, s->p.kk, s->p.kk3);
    for (i = 0; i < 6; i++) t1[i] = xo[i] + K1[i] * dt / 2.0;
    modfn(K2, t1, FF, Mi, s->p.cc, s->p.kk, s->p.kk3);
    for (i = 0; i < 6; i++) t2[i] = xo[i] + K2[i] * dt / 2.0;
    modfn(K3, t2, FF, Mi, s->p.cc, s->p.kk, s->p.kk3);
    for (i = 0; i < 6; i++) t3[i] = xo[i] + K3[i] * dt;
    modfn(K4, t3, FF, Mi, s->p.cc, s->p.kk, s->p.kk3);
    for (i = 0; i < 6; i++) xn[i] = xo[i] + dt * (K1[i] / 6.0 + K2[i] / 3.0 + K3[i] / 3.0 + K4[i] / 6.0);
    if (!s->p.rtcoup) {
        CMP_NP1[0] = s->p.cmposi[0] + xn[0];
        CMP_NP1[1] = s->p.cmposi[1] + xn[1];
        CMP_NP1[2] = s->p.cmroti + xn[2];
        CMV_NP1[0] = xn[3];
        CMV_NP1[1] = xn[4];
        CMV_NP1[2] = xn[5];
        for (i = 0; i < 3; i++) CMA_NP1[i] = (CMV_NP1[i] - CMV_N[i]) / dt;
    } else {
        CMP_NP1[0] = s->p.cmposi[0] + xn[0];
        CMV_NP1[0] = xn[3];
        CMA_NP1[0] = (CMV_NP1[0] - CMV_N[0]) / dt;
        CMP_NP1[1] = s->p.cmposi[1];
        CMV_NP1[1] = 0.0;
        CMA_NP1[1] = 0.0;
        CMP_NP1[2] = s->p.cmroti + xn[0] / rr;
        CMV_NP1[2] = CMV_NP1[0] / rr;
        /* the reference divides the incoming value of its intent(out)
         * argument (cma_np1(3)) by rr here, rigid.F90:296 */
        CMA_NP1[2] = CMA_NP1[2] / rr;
    }
}

/* rigid.F90:373-464 (int_stress): F = sum(-p n + tau) A, moment about cm
 * (the start-of-step centre cmp_n, or the trial centre in the coupling) */
static void int_stress_about(fbo_state *s, const double *centre, double *forcm, double *momcm);
static void int_stress(fbo_state *s, double *forcm, double *momcm)
{
    int_stress_about(s, CMP_N, forcm, momcm);
}

static void int_stress_about(fbo_state *s, const double *centre, double *forcm, double *momcm)
{
    double fyp = 0.0, fzp = 0.0, fyv = 0.0, fzv = 0.0, fy, fz, forgcm[2], mom;
    int i, nlm = s->nlm;
    for (i = 1; i <= nlm; i++) {
        double Fp1 = -s->press[i - 1] * M2(s->lmnor, i, 1) * s->lmA[i - 1];
        double Fp2 = -s->press[i - 1] * M2(s->lmnor, i, 2) * s->lmA[i - 1];
        fyp = fyp + Fp1;
        fzp = fzp + Fp2;
        fyv = fyv + s->tau[2 * (i - 1)] * s->lmA[i - 1];
        fzv = fzv + s->tau[2 * (i - 1) + 1] * s->lmA[i - 1];
    }
    fy = fyp + fyv;
    fz = fzp + fzv;
    forgcm[0] = (1.0 - 1.0 / s->p.rbden) * s->p.rba[0] * s->p.rbgravF[0];
    forgcm[1] = (1.0 - 1.0 / s->p.rbden) * s->p.rba[0] * s->p.rbgravF[1];
    forcm[0] = fy + forgcm[0];
    forcm[1] = fz + forgcm[1];
    *momcm = 0.0;
    for (i = 1; i <= nlm; i++) {
        double r1 = M2(s->lmcc, i, 1) - centre[0], r2 = M2(s->lmcc, i, 2) - centre[1];
        double Ft1 = -s->press[i - 1] * M2(s->lmnor, i, 1) * s->lmA[i - 1] + s->tau[2 * (i - 1)] * s->lmA[i - 1];
        double Ft2 = -s->press[i - 1] * M2(s->lmnor, i, 2) * s->lmA[i - 1] + s->tau[2 * (i - 1) + 1] * s->lmA[i - 1];
        mom = r1 * Ft2 - r2 * Ft1;
        *momcm = *momcm + mom;
    }
    s->forces[0] = s->time;
    s->forces[1] = forcm[0];
    s->forces[2] = forcm[1];
    s->forces[3] = *momcm;
    s->forces[4] = fyp;
    s->forces[5] = fzp;
    s->forces[6] = fyv;
    s->forces[7] = fzv;
}

/* rigid.F90:58-62: constrained coordinates keep their initial kinematics */
static void constrain(fbo_state *s)
{
    for (int i = 0; i < 3; i++)
        if (s->p.rbmcon[i] == 1) {
            CMP_NP1[i] = s->kinori[0][i];
            CMV_NP1[i] = s->kinori[1][i];
            CMA_NP1[i] = s->kinori[2][i];
        }
}

/* rigid.F90:64-126: the markers and vertices moved to the np1 state; commit
 * makes it the new n state (the loose step always commits) */
static void move_body(fbo_state *s, int commit);

/* rigid.F90:4-138 */
int fbo_rigid(fbo_state *s, int ns)
{
    double forcm[2], momcm;
    (void)ns;
    int_stress(s, forcm, &momcm);
    kinem(s, forcm[0], forcm[1], momcm);
    constrain(s);
    move_body(s, 1);
    return FBO_OK;
}

static void move_body(fbo_state *s, int commit)
{
    double r[2][2], cmrot;
    int i, nlm = s->nlm;
    cmrot = CMP_NP1[2] - CMP_N[2];
    get_rotmat(cmrot, r);
    for (i = 1; i <= nlm; i++) {
        double rho[2], c1[2], c2[2], c3[2];
        rho[0] = M2(s->lmcc, i, 1) - CMP_N[0];
        rho[1] = M2(s->lmcc, i, 2) - CMP_N[1];
        c1[0] = -CMV_NP1[2] * rho[1];
        c1[1] = CMV_NP1[2] * rho[0];
        c2[0] = -CMA_NP1[2] * rho[1];
        c2[1] = CMA_NP1[2] * rho[0];
        c3[0] = -CMV_NP1[2] * c1[1];
        c3[1] = CMV_NP1[2] * c1[0];
        M2(s->lmcc, i, 1) = CMP_NP1[0] + (r[0][0] * rho[0] + r[0][1] * rho[1]);
        M2(s->lmcc, i, 2) = CMP_NP1[1] + (r[1][0] * rho[0] + r[1][1] * rho[1]);
        M2(s->lmvel, i, 1) = CMV_NP1[0] + c1[0];
        M2(s->lmvel, i, 2) = CMV_NP1[1] + c1[1];
        M2(s->lmacc, i, 1) = CMA_NP1[0] + c2[0] + c3[0];
        M2(s->lmacc, i, 2) = CMA_NP1[1] + c2[1] + c3[1];
    }
    if (commit)
        for (i = 0; i < 3; i++) {
            CMP_N[i] = CMP_NP1[i];
            CMV_N[i] = CMV_NP1[i];
            CMA_N[i] = CMA_NP1[i];
        }
    /* vertices are rotated about the updated centre (rigid.F90:117-121) */
    for (i = 1; i <= nlm + 1; i++) {
        double rho[2];
        rho[0] = M2(s->vert, i, 1) - CMP_NP1[0];
        rho[1] = M2(s->vert, i, 2) - CMP_NP1[1];
        M2(s->vert, i, 1) = CMP_NP1[0] + (r[0][0] * rho[0] + r[0][1] * rho[1]);
        M2(s->vert, i, 2) = CMP_NP1[1] + (r[1][0] * rho[0] + r[1][1] * rho[1]);
    }
    createnorm(nlm, s->vert, -1.0, s->lmnor);
}

/* ------------------------------------------------ strong coupling
 * No counterpart in the reference, which couples explicitly
 * (main.F90:85-88: fluid_tsch, then rigid).  This restates the strong
 * coupling iteration of fribois2d_b200/csrc/couple.cu on the CPU so that
 * the device's coupled steps have a checker: the step's start state is
 * saved; the body is placed where a trial load moves it (RK4 with the load
 * frozen, as kinem integrates), the fluid step runs from the saved state,
 * its loads are integrated at the trial position (moment about the trial
 * centre), and the trial load is relaxed towards the fluid's with Aitken's
 * factor on the free coordinate q until |F' - F|_q <= tol max(1, |F'_q|).
 * The accepted step commits the body with the fluid's load F'. */

/* save (or restore) the fields, inflow/outflow data and scalars, and/or the
 * body (markers, vertices, normals, centre-of-mass state) */
int fbo_snapshot(fbo_state *s, int save, int fields, int body)
{
    const size_t nf = (size_t)(s->n3 + 1 + 2 * KG) * (size_t)s->n2;
    const size_t nb = (size_t)s->n2 + 2, nlm = (size_t)s->nlm;
    double *fl[] = {s->q2, s->q3, s->pr, s->ru2, s->ru3};
    double *bl[] = {s->qb2s, s->qb2n, s->dqb2s, s->dqb2n, s->qb3s, s->qb3n, s->dqb3s, s->dqb3n,
                    s->dq2x2o, s->dq3x2o};
    double *sc[] = {&s->al, &s->ga, &s->ro, &s->beta, &s->dt, &s->dt_o, &s->time, &s->cflm, &s->q3avg,
                    &s->nbcv, &s->nbcw, &s->ddmin, &s->pravg};
    double *ml[] = {s->lmcc, s->lmvel, s->lmacc, s->lmnor};
    const size_t nfield = 5 * nf + 10 * nb + 13, nbody = 4 * 2 * nlm + 2 * (nlm + 1) + 18;
    size_t off = 0;
    int i;
    if (!s->snap) {
        s->snap = dalloc(nfield + nbody);
        if (!s->snap) return FBO_ERR_INPUT;
    }
#define SNAP(ptr, n)                                                             \
    do {                                                                         \
        if (save) memcpy(s->snap + off, (ptr), sizeof(double) * (n));           \
        else memcpy((ptr), s->snap + off, sizeof(double) * (n));                 \
    } while (0)
    if (fields) {
        for (i = 0; i < 5; i++, off += nf) SNAP(fl[i], nf);
        for (i = 0; i < 10; i++, off += nb) SNAP(bl[i], nb);
        for (i = 0; i < 13; i++, off += 1) SNAP(sc[i], 1);
    } else {
        off += nfield;
    }
    if (body) {
        for (i = 0; i < 4; i++, off += 2 * nlm) SNAP(ml[i], 2 * nlm);
        SNAP(s->vert, 2 * (nlm + 1));
        off += 2 * (nlm + 1);
        SNAP(s->rigid, 18);
    }
#undef SNAP
    return FBO_OK;
}

/* the rigid update split for the coupling: PLACE moves the body to the
 * state the load fin (Fy, Fz, M) gives, without committing; FORCES
 * integrates the loads at that trial state (moment about the trial centre)
 * into the forcecomp row and the np1 state only; COMMIT is the loose update
 * with the load fin */
int fbo_rigid_mode(fbo_state *s, int mode, const double *fin)
{
    double forcm[2], momcm;
    switch (mode) {
    case FBO_RIGID_PLACE:
        kinem(s, fin[0], fin[1], fin[2]);
        constrain(s);
        move_body(s, 0);
        return FBO_OK;
    case FBO_RIGID_FORCES:
        int_stress_about(s, CMP_NP1, forcm, &momcm);
        kinem(s, forcm[0], forcm[1], momcm);
        constrain(s);
        return FBO_OK;
    case FBO_RIGID_COMMIT:
        kinem(s, fin[0], fin[1], fin[2]);
        constrain(s);
        move_body(s, 1);
        return FBO_OK;
    default:
        return FBO_ERR_INPUT;
    }
}

/* one strongly coupled step from the initial guess F0 and relaxation factor
 * omega0 (the caller passes the last Aitken factor of an earlier step,
 * clamped to [0.05, 2], or 0.5 before the first); out: F' (3), fluid
 * solves, relative load residual of the initial guess, converged flag, the
 * last Aitken factor computed in this step (0 if none) */
int fbo_coupled_step(fbo_state *s, int ns, const double F0[3], double tol, int maxit, int q, double omega0,
                     double out[7])
{
    double F[3], Ff[3] = {0.0, 0.0, 0.0}, res[3], rprev[3] = {0.0, 0.0, 0.0}, omega = omega0, res0 = 0.0;
    double aitken = 0.0;
    int it, i, conv = 0, st;
    fbo_snapshot(s, 1, 1, 1);
    for (i = 0; i < 3; i++) F[i] = F0[i];
    for (it = 0; it < maxit; it++) {
        if (it > 0) fbo_snapshot(s, 0, 1, 1);
        fbo_rigid_mode(s, FBO_RIGID_PLACE, F);
        st = fbo_fluid_tsch(s, ns);
        if (st) return st;
        fbo_rigid_mode(s, FBO_RIGID_FORCES, NULL);
        for (i = 0; i < 3; i++) {
            Ff[i] = s->forces[1 + i];
            res[i] = Ff[i] - F[i];
        }
        if (it == 0) res0 = fabs(res[q]) / fmax(1.0, fabs(Ff[q]));
        conv = fabs(res[q]) <= tol * fmax(1.0, fabs(Ff[q]));
        if (conv) break;
        if (it > 0) {
            const double dr = res[q] - rprev[q];
            if (dr != 0.0) {
                omega = -omega * rprev[q] / dr;
                aitken = omega;
            }
        }
        for (i = 0; i < 3; i++) {
            F[i] = F[i] + omega * res[i];
            rprev[i] = res[i];
        }
    }
    /* accept: body back to the start of the step, then the update with F' */
    fbo_snapshot(s, 0, 0, 1);
    for (i = 0; i < 3; i++) s->forces[1 + i] = Ff[i];
    fbo_rigid_mode(s, FBO_RIGID_COMMIT, Ff);
    s->time = s->time + s->dt;
    s->dt_o = s->dt;
    for (i = 0; i < 3; i++) out[i] = Ff[i];
    out[3] = (double)(conv ? it + 1 : it);
    out[4] = res0;
    out[5] = (double)conv;
    out[6] = aitken;
    return FBO_OK;
}

/* ------------------------------------------------------------ drivers */

int fbo_set_substep(fbo_state *s, int ns, int n)
{
    if (s->p.nsst == 3) {
        s->al = s->alm[n - 1];
        s->ga = s->gam[n - 1];
        s->ro = s->rom[n - 1];
    } else {
        if (ns == 0) {
            s->ga = 1.0;
            s->ro = 0.0;
        } else {
            s->ga = 1.0 + 0.5 * s->dt / s->dt_o;
            s->ro = -0.5 * s->dt / s->dt_o;
        }
        s->al = s->ga + s->ro;
    }
    s->beta = s->dt / s->ren * 0.5;
    return FBO_OK;
}

int fbo_stage(fbo_state *s, int stage, int n)
{
    int st = FBO_OK;
    switch (stage) {
    case FBO_ST_CFL: cfl(s); break;
    case FBO_ST_BOUCDQ: boucdq(s); break;
    case FBO_ST_HDNL2: hdnl2(s); break;
    case FBO_ST_HDNL3: hdnl3(s); break;
    case FBO_ST_INVTR2: invtr2(s); break;
    case FBO_ST_INVTR3: invtr3(s); break;
    case FBO_ST_LGRDIST: st = lgrdistribution(s); break;
    case FBO_ST_FORCING: st = forcing_mls(s, n); break;
    case FBO_ST_HELSOLVE: helsolve(s); break;
    case FBO_ST_DIVG: divg(s); break;
    case FBO_ST_PHCALC: phcalc(s); break;
    case FBO_ST_UPDVP: updvp(s); break;
    case FBO_ST_PRCALC: prcalc(s); break;
    case FBO_ST_PRSUBMEAN: pr_submean(s); break;
    case FBO_ST_BOUCQT: boucqt(s); break;
    case FBO_ST_CHECKBCS: checkbcs(s); break;
    case FBO_ST_LOADS: st = loads_transfer(s); break;
    case FBO_ST_RIGID: st = fbo_rigid(s, 0); break;
    case FBO_ST_SOLQ2J: solq2j(s); break;
    case FBO_ST_SOLQ2K: solq2k(s); break;
    case FBO_ST_SOLQ3J: solq3j(s); break;
    case FBO_ST_SOLQ3K: solq3k(s); break;
    default: st = FBO_ERR_INPUT;
    }
    if (st != FBO_OK && s->status == FBO_OK) s->status = st;
    return st;
}

/* fluid_tsch.F90:4-204 */
int fbo_fluid_tsch(fbo_state *s, int ns)
{
    int n, st;
    cfl(s);
    if (!s->p.idtv) {
        if (ns == 0) {
            s->cflm = s->cflm * s->dt;
        } else {
            s->dt = s->p.cflmax / s->cflm;
            if (s->dt > s->p.dtmax) s->dt = s->p.dtmax;
        }
        if (s->dt < 1.0e-8) return s->status = FBO_ERR_CFL;
    } else {
        s->cflm = s->cflm * s->dt;
        if (s->cflm > s->p.cfllim) return s->status = FBO_ERR_CFL;
    }
    s->beta = s->dt / s->ren * 0.5;
    for (n = 1; n <= s->p.nsst; n++) {
        fbo_set_substep(s, ns, n);
        boucdq(s);
        hdnl2(s);
        hdnl3(s);
        invtr2(s);
        invtr3(s);
        if (s->p.ibact) {
            if (n == 1) {
                st = lgrdistribution(s);
                if (st) return s->status = st;
            }
            st = forcing_mls(s, n);
            if (st) return s->status = st;
        }
        helsolve(s);
        divg(s);
        phcalc(s);
        updvp(s);
        prcalc(s);
        pr_submean(s);
        boucqt(s);
    }
    if (s->p.ibact) checkbcs(s);
    if (s->p.ibact && s->p.cbody) {
        st = loads_transfer(s);
        if (st) return s->status = st;
    }
    return FBO_OK;
}

/* main.F90:85-97: one time step including the rigid update and the clock */
int fbo_step(fbo_state *s, int ns)
{
    int st = fbo_fluid_tsch(s, ns);
    if (st) return st;
    if (s->p.ibact) fbo_rigid(s, ns);
    s->time = s->time + s->dt;
    s->dt_o = s->dt;
    return FBO_OK;
}

int fbo_status(fbo_state *s) { return s->status; }

double *fbo_array(fbo_state *s, int id, long *n)
{
    long nf = (long)s->n2 * (long)(s->n3 + 1 + 2 * KG);
    long n1 = s->n2 + 2, n3 = s->n3 + 2;
    switch (id) {
#define R(ID, ptr, cnt) case ID: *n = (cnt); return (ptr)
    R(FBO_Q2, s->q2, nf); R(FBO_Q3, s->q3, nf); R(FBO_PR, s->pr, nf); R(FBO_DPH, s->dph, nf);
    R(FBO_Q2F, s->q2f, nf); R(FBO_Q3F, s->q3f, nf); R(FBO_RHS, s->rhs, nf);
    R(FBO_RHS2, s->rhs2, nf); R(FBO_RHS3, s->rhs3, nf); R(FBO_RU2, s->ru2, nf);
    R(FBO_RU3, s->ru3, nf); R(FBO_QCAP, s->qcap, nf); R(FBO_FEY, s->fey, nf); R(FBO_FEZ, s->fez, nf);
    R(FBO_QB2S, s->qb2s, n1); R(FBO_QB2N, s->qb2n, n1); R(FBO_DQB2S, s->dqb2s, n1);
    R(FBO_DQB2N, s->dqb2n, n1); R(FBO_QB3S, s->qb3s, n1); R(FBO_QB3N, s->qb3n, n1);
    R(FBO_DQB3S, s->dqb3s, n1); R(FBO_DQB3N, s->dqb3n, n1); R(FBO_DQ2X2O, s->dq2x2o, n1);
    R(FBO_DQ3X2O, s->dq3x2o, n1);
    R(FBO_RC, s->rc, n1); R(FBO_RM, s->rm, n1); R(FBO_ZZ, s->zz, n3); R(FBO_ZM, s->zm, n3);
    R(FBO_G2RC, s->g2rc, n1); R(FBO_G2RM, s->g2rm, n1); R(FBO_G3RC, s->g3rc, n3);
    R(FBO_G3RM, s->g3rm, n3); R(FBO_UDX2C, s->udx2c, n1); R(FBO_UDX2M, s->udx2m, n1);
    R(FBO_UDX3C, s->udx3c, n3); R(FBO_UDX3M, s->udx3m, n3);
    R(FBO_AM2J, s->am2j, n1); R(FBO_AC2J, s->ac2j, n1); R(FBO_AP2J, s->ap2j, n1);
    R(FBO_AM3J, s->am3j, n1); R(FBO_AC3J, s->ac3j, n1); R(FBO_AP3J, s->ap3j, n1);
    R(FBO_AM3CK, s->am3ck, n3); R(FBO_AC3CK, s->ac3ck, n3); R(FBO_AP3CK, s->ap3ck, n3);
    R(FBO_AM3SK, s->am3sk, n3); R(FBO_AC3SK, s->ac3sk, n3); R(FBO_AP3SK, s->ap3sk, n3);
    R(FBO_AMPHJ, s->amphj, n1); R(FBO_ACPHJ, s->acphj, n1); R(FBO_APPHJ, s->apphj, n1);
    R(FBO_AMPHK, s->amphk, n3); R(FBO_ACPHK, s->acphk, n3); R(FBO_APPHK, s->apphk, n3);
    R(FBO_WR, s->wr, s->n3m); R(FBO_ZMM, s->zmm, (long)s->n3m * s->n3m);
    R(FBO_ZMMT, s->zmmt, (long)s->n3m * s->n3m);
    R(FBO_LMCC, s->lmcc, 2L * s->nlm); R(FBO_LMVEL, s->lmvel, 2L * s->nlm);
    R(FBO_LMACC, s->lmacc, 2L * s->nlm); R(FBO_LMNOR, s->lmnor, 2L * s->nlm);
    R(FBO_LMA, s->lmA, s->nlm); R(FBO_VERT, s->vert, 2L * (s->nlm + 1));
    R(FBO_PHI, s->phi, 18L * s->nlm); R(FBO_CL, s->cl, 2L * s->nlm);
    R(FBO_PRESS, s->press, s->nlm); R(FBO_TAU, s->tau, 2L * s->nlm);
    R(FBO_BCERRV, s->bcerrv, s->nlm); R(FBO_BCERRW, s->bcerrw, s->nlm);
    R(FBO_RIGID, s->rigid, 18); R(FBO_FORCES, s->forces, 8);
#undef R
    case FBO_SCALARS:
        s->scalars[0] = s->time; s->scalars[1] = s->dt; s->scalars[2] = s->dt_o;
        s->scalars[3] = s->beta; s->scalars[4] = s->al; s->scalars[5] = s->ga;
        s->scalars[6] = s->ro; s->scalars[7] = s->cflm; s->scalars[8] = s->q3avg;
        s->scalars[9] = s->nbcv; s->scalars[10] = s->nbcw; s->scalars[11] = s->ddmin;
        s->scalars[12] = s->pravg;
        *n = 13;
        return s->scalars;
    }
    *n = 0;
    return NULL;
}

int *fbo_iarray(fbo_state *s, int id, long *n)
{
    switch (id) {
    case FBO_LMIND: *n = 4L * s->nlm; return s->lmind;
    case FBO_EULINS: *n = 36L * s->nlm; return s->eulins;
    case FBO_JMV: *n = s->n2 + 2; return s->jmv;
    case FBO_JPV: *n = s->n2 + 2; return s->jpv;
    case FBO_KMV: *n = s->n3 + 2; return s->kmv;
    case FBO_KPV: *n = s->n3 + 2; return s->kpv;
    }
    *n = 0;
    return NULL;
}
