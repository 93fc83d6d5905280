// Strong fluid-structure coupling iterated on the device (definitions in
// couple.cu).  No counterpart in the reference, which couples explicitly
// (src/main.F90:85-88: fluid_tsch, then rigid); the *_o save arrays and the
// fsicoup parameters of src/declarations.F90:271-278 show the intent.
#pragma once

#include <cuda_runtime.h>

#include "../../include/fribois2d.h"
#include "device.cuh"

namespace fb {

constexpr int kCplHist = 16;   // converged steps kept per case for the predictors
constexpr int kCplDepth = 8;   // steps of history in the learned predictor's features
constexpr int kCplIn = 27;     // 3 x kCplDepth second differences + Re, mass ratio, reduced velocity
constexpr int kCplOut = 2;     // corrections of the displacement and the load
constexpr int kCplH = 64;      // hidden width of the perceptron (as in mlp.cu)
constexpr int kSnapMax = 24;   // arrays in one case's saved state

// One case's coupling: set-up, iteration state, converged history, statistics.
struct Couple {
    double tol, omega0;
    int maxit, q, learned, cap;        // q: the free body coordinate; cap: sample ring size
    double feat_re, feat_mr, feat_ur;  // the case parameters among the features
    const float *mlp;                  // perceptron parameters [W1 b1 W2 b2 W3 b3] or null
    const float *norm;                 // x mean[27], x std[27], t mean[2], t std[2]
    double *forces;                    // the case's forcecomp row
    const double *rigid;               // the case's centre-of-mass state
    float *sx, *st;                    // training samples: cap x kCplIn, cap x kCplOut
    double F[3], Ff[3], rprev[3], omega;
    double omega_last;                 // the last Aitken factor computed (warm start of the next step)
    double fin[4];                     // trial (or accepted) load handed to k_rigid; [3] = solves
    int it, active, conv, have_omega;
    int nh, spare2;                    // converged steps in hp/hv/hf, oldest first
    double hp[kCplHist][3], hv[kCplHist][3], hf[kCplHist][3];
    double steps, solves, maxit_hits, res0;
    unsigned long long nsamples;       // samples written (ring slot = nsamples % cap)
};

// One case's saved state: entries [0, nfield) are the fluid state (fields,
// inflow/outflow data, scalars), the rest the body (markers, vertices,
// centre-of-mass state).
struct SnapList {
    int n, nfield;
    double *arr[kSnapMax];
    double *copy[kSnapMax];
    long len[kSnapMax];
    const Couple *c;                   // the in-loop restore runs while c is iterating
};

enum SnapMode { SNAP_SAVE = 0, SNAP_RESTORE_LOOP = 1, SNAP_RESTORE_BODY = 2 };

// n cases: a device array of n Couple pointers / n SnapLists
void launch_couple_begin(Couple *const *c, int n, cudaStream_t s);
void launch_snap(const SnapList *l, int n, int mode, long longest, cudaStream_t s);
// set_cond: write `any case still iterating` into the graph conditional h;
// any_out (device, may be null): the same flag for a host-driven loop
void launch_couple_update(Couple *const *c, int n, cudaGraphConditionalHandle h, int set_cond, int *any_out,
                          cudaStream_t s);
void launch_couple_accept(Couple *const *c, int n, cudaStream_t s);
void launch_couple_record(Couple *const *c, int n, cudaStream_t s);

// the perceptron's parameters in device memory (mlp.cu): [W1 b1 W2 b2 W3 b3]
const float *mlp_params_device(const fb_mlp *m, int *n_in, int *n_out);

}  // namespace fb
