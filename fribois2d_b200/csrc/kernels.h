// Kernel launchers of the fluid time step (definitions in kernels.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "device.cuh"

namespace fb {

constexpr int kRedSlot = 65536;  // block partials per reduction slot

cudaError_t kernels_configure();   // shared-memory limits (once per device)
void launch_cfl(const Dev &d, cudaStream_t s);
void launch_boucdq(const Dev &d, double ga, double ro, cudaStream_t s);
// TMA descriptors of the fields that the stencil tiles stage (q2, q3, pr for
// k_nl_rhs, dph for k_updvp_prcalc): 2-D arrays (j - 1 fastest, row k,
// k = 0 .. n3), one box per tile and field
struct alignas(64) NlMaps {
    CUtensorMap q2, q3, pr, dph;
};
int encode_nl_maps(NlMaps *m, const Dev &d);   // FB_OK, or an error (no maps)
// pend / deferred: the fused step's deferred pr_submean of RK3 substeps 1 and 2.
// maps: stage the tiles with TMA (the single-case step); null: cp.async
void launch_nl_rhs(const Dev &d, double al, double ga, double ro, cudaStream_t s, bool pend = false,
                   const NlMaps *maps = nullptr);
void launch_lgrdist(const Dev &d, cudaStream_t s);
void launch_mls_setup(const Dev &d, cudaStream_t s);
void launch_mls_interp(const Dev &d, cudaStream_t s);
void launch_mls_spread(const Dev &d, cudaStream_t s);
void launch_spread_chains(const Dev &d, cudaStream_t s);
void launch_helsolve(const Dev &d, const SubDev &sd, cudaStream_t s);
// rmax (may be null): n2m row maxima of |dph| accumulated for the INT8 digit cut
void launch_divg(const Dev &d, double usdtal, cudaStream_t s, double *rmax = nullptr);
void launch_updvp_prcalc(const Dev &d, double al, double be, cudaStream_t s, bool pend = false,
                         const NlMaps *maps = nullptr);
// mbox[0] = *d.status, mbox[1..8] = d.forces[0..7] (when forces); mbox in
// mapped host memory
void launch_publish(const Dev &d, bool forces, double *mbox, cudaStream_t s);
void launch_submean_boucqt(const Dev &d, cudaStream_t s, bool deferred = false);
void launch_substep_mid(const Dev &d, int slot, double ga, double ro, cudaStream_t s);  // boucqt + next boucdq
void launch_loads(const Dev &d, cudaStream_t s);
void launch_diag(const Dev &d, int hist_rows, cudaStream_t s);
enum RigidMode { RIGID_STEP = 0, RIGID_PLACE = 1, RIGID_FORCES = 2, RIGID_COMMIT = 3 };
// mbox (mapped host memory, may be null; RIGID_STEP and RIGID_COMMIT): the status
// word and the forcecomp row, written at the end as k_publish does
void launch_rigid(const Dev &d, int hist_rows, cudaStream_t s, int mode = RIGID_STEP, const double *fin = nullptr,
                  double *mbox = nullptr);

// grouped forms (one launch over a group of cases; substep n 0-based)
void glaunch_cfl(const Group &g, cudaStream_t s);
void glaunch_boucdq(const Group &g, int n, cudaStream_t s);
void glaunch_nl_rhs(const Group &g, int n, cudaStream_t s, bool pend = false);
void glaunch_marker_setup(const Group &g, cudaStream_t s);   // lgrdist, MLS weights, spreading chains
void glaunch_forcing(const Group &g, cudaStream_t s);        // interpolation and spreading
void glaunch_divg(const Group &g, int n, cudaStream_t s);
void glaunch_updvp_prcalc(const Group &g, int n, cudaStream_t s, bool pend = false);
void glaunch_submean_boucqt(const Group &g, cudaStream_t s, bool deferred = false);
void glaunch_substep_mid(const Group &g, int n_next, int slot, cudaStream_t s);
void glaunch_loads(const Group &g, cudaStream_t s);
void glaunch_rigid(const Group &g, cudaStream_t s, int mode = RIGID_STEP);
void glaunch_diag(const Group &g, cudaStream_t s);

}  // namespace fb
