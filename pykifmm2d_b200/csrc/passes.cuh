// passes.cuh -- arguments shared by the pass kernels.
#pragma once
#include "kifmm_internal.cuh"

namespace kifmm {

struct PassArgs {
    LevelTable T;
    int Q, kind;
    double k;
    double root, W;
    const double *ops;
    const float *ops_f;
    size_t stride, off_inv, off_m2m, off_l2l, off_m2l, off_large;
    const uint64_t *ent;
    const int32_t *ent_node;
    const uint64_t *nkey;
    const int8_t *nlev;
    const uint8_t *nflag;
    const int32_t *nbot, *ntop, *nchild, *nent, *ncoll;
    const double *xs, *ys, *taus;
    double *pots;
    double *uup, *udown;
    const double *taylor;  // Laplace L2P coefficients map, or null
    const float *taylor_f;  // FP32 copy of it (the orders computed in FP32)
};

// Node centre, exactly the reference's xmid = xmin + w/2 (tree.py:339-346):
// both are dyadic numbers inside the checked coordinate range.
__device__ __forceinline__ void node_center(const PassArgs &A, int g, int l, double &cx, double &cy) {
    uint64_t k = A.nkey[g];
    double w = ldexp(A.W, -l);
    cx = A.root + ((double)compact2(k >> 1) + 0.5) * w;
    cy = A.root + ((double)compact2(k) + 0.5) * w;
}

PassArgs make_pass_args(kifmm_plan *P);
// passes_mixed.cu
void run_passes_mixed(kifmm_plan *P);
void run_eval_sources_mixed(kifmm_plan *P, int check_self);
void run_eval_targets_mixed(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self,
                            double *pot);

}  // namespace kifmm
