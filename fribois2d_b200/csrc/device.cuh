// Device view of one case: plain pointers and scalars passed by value to
// every kernel.  Fields are stored k-major with row pitch P (doubles):
// element (j, k) of a reference array A(j, k), j = 1..n2, k = 0..n3, lives
// at A[k*P + (j-1)].  One-dimensional arrays keep the reference's 1-based
// indexing (index 0 unused).
#pragma once

#include <cstdint>

namespace fb {

constexpr int kSD = 9;  // MLS support nodes per marker and direction (dimSD)

struct TriDev {          // factors of one tridiagonal system (DGTTRF output)
    int n;
    int pivoted;
    const double *dl, *dinv, *du, *du2;
    const int *ipiv;     // 1-based pivot rows as LAPACK returns them
};

struct ScanSys {         // LU substitution as two recurrences (tri.cu)
    const double *a, *e, *g;  // y(i) = a(i) y(i-1) + b(i);  x(i) = e(i) x(i+1) + g(i) y(i)
};

struct SubDev {          // substep constants (fluid_tsch.F90:64-77)
    double al, ga, ro, beta, betadx, usdtal, ugkks, ugkkn;
    const double *by2, *bz2, *by3, *bz3;  // row normalisers 1/(1 - betadx*ac), 1-based
    TriDev y2, z2, y3, z3;                // solq2j, solq2k, solq3j, solq3k systems
    ScanSys sy2, sz2, sy3, sz3;           // the same systems for the scan solver
    int scan_ok;                          // 0 if a system needed row interchanges
    int win_y, win_z;                     // truncation windows (y, z) of the windowed helsolve; 0 = off
    int win_tk;                           // its tile height in k (32 or 64; set by the autotuner)
};

struct Dev {
    int n2, n3, n2m, n3m, P, NK, nlm, nsst, wfun, ldh;
    int indz;                // getintvort line (utils_proc.F90:607-609); 0 = none
    int vardt;               // idtv = .false.: dt follows the CFL number (no fixed-dt check)
    double dx2, dx3, dx2q, dx3q, ren, visc, dt, cou, q3uw, q3lw, rext2, alx3;
    double radiusSD, kprobe, ddmin, area_out, cfllim;
    // grid (1-based)
    const double *rc, *rm, *zz, *zm, *g2rc, *g2rm, *g3rc, *g3rm, *udx2c, *udx2m, *udx3c, *udx3m;
    const int *jmv, *jpv, *kmv, *kpv;
    const double *am2j, *ac2j, *ap2j, *am3j, *ac3j, *ap3j;
    const double *am3ck, *ac3ck, *ap3ck, *am3sk, *ac3sk, *ap3sk;
    const double *amphj, *acphj, *apphj, *amphk, *acphk, *apphk;
    // Poisson: reciprocal pivots of each mode's y system, [mode][j] pitch ldh
    const double *pg;
    // fields
    double *q2, *q3, *pr, *dph, *rhs2, *rhs3, *ru2, *ru3, *hmn;
    // inflow / outflow (1-based)
    double *qb2s, *qb2n, *dqb2s, *dqb2n, *qb3s, *qb3n, *dqb3s, *dqb3n, *dq2x2o, *dq3x2o;
    // markers
    double *lmcc, *lmvel, *lmacc, *lmnor, *lmA, *vert;
    int *lmind;              // [marker][dir][2]
    int *eulins;             // [marker][dir][2][kSD]
    double *phi, *cl;        // [marker][dir][kSD], [marker][dir]
    double *contrib;         // [marker][dir][kSD] forcing contributions of one substep
    int *bcnt, *bucket;      // markers per support-box start cell, [dir][cell] and [dir][cell][bcap]
    int bcap;
    int *chain;              // per contribution slot: next slot of the same cell in marker
                             // order (>= 0) or -1 at the end, written by the cell's head
    int *chead;              // per contribution slot: 1 if it heads its cell's chain
    double *probe;           // [marker][24]: ucy(7), ucz(7), pc(7), tan(2), flag
    double *press, *tau, *bcerrv, *bcerrw;
    // rigid body
    double *rigid;           // cmp_n, cmv_n, cma_n, cmp_np1, cmv_np1, cma_np1
    double *forces;          // forcecomp.out row
    double *scal;            // see Scal
    double *hist;            // history rows, FB_HIST_COLS each
    double *red;             // block partial sums
    unsigned *count;         // last-block counters
    int *status;
    double rbden, rba0, rba1, cmposi0, cmposi1, cmroti, rbgravF0, rbgravF1, rrr;
    double kk[3], kk3[3], cc[3], kinori[9];
    int rbmcon[3], rtcoup;
};

// device scalar slots
enum Scal {
    S_TIME = 0, S_CFLM, S_Q3AVG, S_NBCV, S_NBCW, S_PRAVG, S_QOUT, S_DT, S_STEP, S_CFLRAW, S_COUNT
};

__host__ __device__ inline size_t fidx(const Dev &d, int j, int k) {
    return static_cast<size_t>(k) * static_cast<size_t>(d.P) + static_cast<size_t>(j - 1);
}

}  // namespace fb
