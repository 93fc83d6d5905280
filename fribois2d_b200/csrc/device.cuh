// Device view of one case: plain pointers and scalars passed by value to
// every kernel.  Fields are stored k-major with row pitch P (doubles):
// element (j, k) of a reference array A(j, k), j = 1..n2, k = 0..n3, lives
// at A[k*P + (j-1)].  One-dimensional arrays keep the reference's 1-based
// indexing (index 0 unused).
#pragma once

#include <cstdint>

namespace fb {

constexpr int kSD = 9;  // MLS support nodes per marker and direction (dimSD)
constexpr int kBucket = 16;        // marker slots per spreading-table entry
constexpr int kBucketLevels = 16;  // entries per start cell at most (256 boxes)
constexpr int kHeadList = 8;       // chain members a head keeps in line (read with two 16-byte loads)

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
    // support-box start cell -> markers: an open-addressing table of 2^hlog
    // entries (sized by the marker count), each a key ((dir, cell) x
    // kBucketLevels + level, plus one; 0 = empty), a count and kBucket marker
    // slots; a cell with more than kBucket boxes continues at the next level
    unsigned long long *hkey;
    int *hcnt, *hval;
    int *hslot;              // per (marker, dir): its entry plus one, 0 = none
    int hlog;
    int *chain;              // per contribution slot: next slot of the same cell in marker
                             // order (>= 0) or -1 at the end, written by the cell's head
    int *chead;              // per contribution slot: 1 if it heads its cell's chain
    int *hlist;              // per head slot: the chain's next kHeadList slots in order (then chain[])
    int *hlen;               // per head slot: the chain's length after the head
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

// One case of a grouped launch: cases of one launch geometry are stepped by
// single launches whose blockIdx.z selects the case; each block reads its
// case's view and substep constants from a device array of these.
constexpr int kMaxSub = 3;
struct GroupCase {
    Dev d;
    SubDev s[kMaxSub];
    int hist_rows;
    // strongly coupled batches: the case takes part in a launch only while
    // *gate is non-zero (null: always); fin is its trial load for k_rigid
    const int *gate;
    const double *fin;
};

#ifdef __CUDACC__
// asynchronous 8-byte global -> shared copies (no register round trip, all
// of a thread's copies in flight at once); cp_wait completes this thread's
// copies, a barrier then publishes them to the block
__device__ __forceinline__ void cp8(double *dst, const double *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// *addr = max(*addr, v) for non-negative, non-NaN doubles: their bit
// patterns order as their values
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// copies case blockIdx.z's view of a group (and the constants of substep n
// when ss is given) to shared memory, then waits for the preceding kernel
// (programmatic dependent launch) and the block.  The group array is written
// once by the host, so the copy may run before the grid dependency wait.
template <class T>
__device__ __forceinline__ void copy_words(const T &src, T *dst, int t, int nt) {
    static_assert(sizeof(T) % 8 == 0, "copied in 8-byte words");
    const unsigned long long *s = reinterpret_cast<const unsigned long long *>(&src);
    unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
    for (int i = t; i < static_cast<int>(sizeof(T) / 8); i += nt) d[i] = __ldg(s + i);
}
// Returns false when the case sits out this launch (its coupling iteration
// has converged): the whole block then returns at once.
__device__ __forceinline__ bool stage_case(const GroupCase *__restrict__ g, Dev *sd, SubDev *ss = nullptr,
                                           int n = 0, bool gated = true) {
    const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nt = blockDim.x * blockDim.y * blockDim.z;
    copy_words(g[blockIdx.z].d, sd, t, nt);
    if (ss) copy_words(g[blockIdx.z].s[n], ss, t, nt);
    asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory");
    __syncthreads();
    const int *gate = g[blockIdx.z].gate;   // written by earlier kernels: read after the wait
    return !gated || !gate || *gate != 0;
}
#endif

// Host view of a launch group: cases whose launches have one geometry (grid
// sizes, marker count, helsolve tiles), stepped by launches with gridDim.z = n.
struct Group {
    const GroupCase *cases;  // device array of n
    int n;
    Dev rep;                 // the first case: launch geometry only
    int win_tk;              // windowed helsolve tile height
    int win_ky[kMaxSub], win_kz[kMaxSub];  // largest windows of the group per substep
};

// device scalar slots
enum Scal {
    S_TIME = 0, S_CFLM, S_Q3AVG, S_NBCV, S_NBCW, S_PRAVG, S_QOUT, S_DT, S_STEP, S_CFLRAW, S_COUNT,
    // transient within a step (not part of the saved state): the pressure
    // means of RK3 substeps 1 and 2 while their subtraction is deferred
    S_PRAVG1 = S_COUNT, S_PRAVG2, S_SLOTS
};

__host__ __device__ inline size_t fidx(const Dev &d, int j, int k) {
    return static_cast<size_t>(k) * static_cast<size_t>(d.P) + static_cast<size_t>(j - 1);
}

}  // namespace fb
