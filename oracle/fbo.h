/*
 * CPU oracle for the FRiBoIS2D fluid time step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, loop-for-loop restatement of the reference's hot path
 * (src/fluid_tsch.F90 and everything it calls, plus src/rigid.F90) used as
 * the parity checker for the CUDA implementation and as the timed CPU
 * baseline.  It is never linked into the product library.
 *
 * Parity status: UNPINNED against the reference binary.  The reference is
 * Fortran/MPI and cannot be built here (no Fortran compiler, no MPI, no
 * system LAPACK); it ships no tests or golden vectors.  The LAPACK pieces
 * the reference calls (DGEEV/DGESV at set-up, DGTTRF/DGTTRS per line,
 * DGEMM) are pinned against scipy's LAPACK by the tests, and the whole
 * step is cross-checked against an independent NumPy/LAPACK restatement.
 *
 * Layout follows the reference: every field is column-major A(j,k), j the
 * contiguous y index 1..n2, k the z index with the reference's ghost rows
 * (-2..n3+2 on one rank).  Marker arrays are row-major [marker][component].
 */
#ifndef FBO_H
#define FBO_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fbo_params {
    int n2, n3, nsst, idtv, ibact, cbody, wfun, forst, inslws, inslwn, rtcoup, nlm;
    int rbmcon[3];
    double alx3, rext2, dt, dtmax, cflmax, cfllim, resid, cou, visc, q3uw, q3lw;
    double kprobe, radiusSD;
    double rbden, rba[2], cmposi[2], cmroti, rbgravF[2], kk[3], kk3[3], cc[3], rrr, ipert[3];
} fbo_params;

typedef struct fbo_state fbo_state;

/* status codes, numerically identical to the product's FB_* codes */
enum {
    FBO_OK = 0,
    FBO_ERR_CFL = 1,          /* fluid_tsch.F90:43-55 */
    FBO_ERR_MLS = 2,          /* MLSint.F90:157-163, 248-255 */
    FBO_ERR_MARKER_OUT = 3,   /* lgrdistribution.F90:217-221 */
    FBO_ERR_INPUT = 4
};

/* array ids for fbo_array() */
enum {
    FBO_Q2 = 0, FBO_Q3, FBO_PR, FBO_DPH, FBO_Q2F, FBO_Q3F, FBO_RHS, FBO_RHS2, FBO_RHS3,
    FBO_RU2, FBO_RU3, FBO_QCAP, FBO_FEY, FBO_FEZ,                       /* fields */
    FBO_QB2S = 20, FBO_QB2N, FBO_DQB2S, FBO_DQB2N, FBO_QB3S, FBO_QB3N, FBO_DQB3S,
    FBO_DQB3N, FBO_DQ2X2O, FBO_DQ3X2O,                                  /* n2+1 */
    FBO_RC = 40, FBO_RM, FBO_ZZ, FBO_ZM, FBO_G2RC, FBO_G2RM, FBO_G3RC, FBO_G3RM,
    FBO_UDX2C, FBO_UDX2M, FBO_UDX3C, FBO_UDX3M,
    FBO_AM2J, FBO_AC2J, FBO_AP2J, FBO_AM3J, FBO_AC3J, FBO_AP3J,
    FBO_AM3CK, FBO_AC3CK, FBO_AP3CK, FBO_AM3SK, FBO_AC3SK, FBO_AP3SK,
    FBO_AMPHJ, FBO_ACPHJ, FBO_APPHJ, FBO_AMPHK, FBO_ACPHK, FBO_APPHK,   /* 1-based, n+1 */
    FBO_WR = 80, FBO_ZMM, FBO_ZMMT,                                     /* n3m, n3m^2 */
    FBO_LMCC = 90, FBO_LMVEL, FBO_LMACC, FBO_LMNOR, FBO_LMA, FBO_VERT,
    FBO_PHI, FBO_CL, FBO_PRESS, FBO_TAU, FBO_BCERRV, FBO_BCERRW,
    FBO_RIGID = 110,   /* cmp_n,cmv_n,cma_n,cmp_np1,cmv_np1,cma_np1 (18) */
    FBO_SCALARS = 111, /* time,dt,dt_o,beta,al,ga,ro,cflm,q3avg,nbcv,nbcw,ddmin,pravg */
    FBO_FORCES = 112   /* forcecomp.out row: time,Fy,Fz,M,Fyp,Fzp,Fyv,Fzv */
};
enum { FBO_LMIND = 0, FBO_EULINS = 1, FBO_JMV, FBO_JPV, FBO_KMV, FBO_KPV };

/* stage ids for fbo_stage(): one per reference subroutine */
enum {
    FBO_ST_CFL = 0, FBO_ST_BOUCDQ, FBO_ST_HDNL2, FBO_ST_HDNL3, FBO_ST_INVTR2, FBO_ST_INVTR3,
    FBO_ST_LGRDIST, FBO_ST_FORCING, FBO_ST_HELSOLVE, FBO_ST_DIVG, FBO_ST_PHCALC,
    FBO_ST_UPDVP, FBO_ST_PRCALC, FBO_ST_PRSUBMEAN, FBO_ST_BOUCQT, FBO_ST_CHECKBCS,
    FBO_ST_LOADS, FBO_ST_RIGID, FBO_ST_SOLQ2J, FBO_ST_SOLQ2K, FBO_ST_SOLQ3J, FBO_ST_SOLQ3K
};

fbo_state *fbo_create(const fbo_params *p, const double *ycoord, const double *zcoord,
                      const double *vert);
void fbo_destroy(fbo_state *s);
/* eigen data of the z Poisson operator (phini.F90:75-92), n3m and n3m x n3m column-major */
void fbo_set_eigen(fbo_state *s, const double *wr, const double *zmm, const double *zmmt);
double *fbo_array(fbo_state *s, int id, long *n);
int *fbo_iarray(fbo_state *s, int id, long *n);
int fbo_fluid_tsch(fbo_state *s, int ns);       /* fluid_tsch.F90:4-204 */
int fbo_rigid(fbo_state *s, int ns);            /* rigid.F90:4-138 */
int fbo_step(fbo_state *s, int ns);             /* main.F90:85-97 */
int fbo_set_substep(fbo_state *s, int ns, int n);
int fbo_stage(fbo_state *s, int stage, int n);
int fbo_status(fbo_state *s);
/* strong coupling (no reference counterpart): see fbo.c */
enum { FBO_RIGID_PLACE = 1, FBO_RIGID_FORCES = 2, FBO_RIGID_COMMIT = 3 };
int fbo_snapshot(fbo_state *s, int save, int fields, int body);
int fbo_rigid_mode(fbo_state *s, int mode, const double *fin);
int fbo_coupled_step(fbo_state *s, int ns, const double F0[3], double tol, int maxit, int q, double omega0,
                     double out[7]);
/* LAPACK restatements, exported so the tests can pin them against LAPACK */
int fbo_dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv);
void fbo_dgtts2(int n, const double *dl, const double *d, const double *du, const double *du2,
                const int *ipiv, double *b);
void fbo_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
