// passes.cuh -- arguments shared by the pass kernels.
#pragma once
#include "kifmm_internal.cuh"

namespace kifmm {

struct PassArgs {
    LevelTable T;
    int Q, kind;   // Q: state length per node (2 Nequiv for complex values)
    int Qc;        // points per circle (Nequiv)
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
    const int32_t *leaf_rec;  // [n_leaf_list][LEAF_REC_WORDS] leaf records (build_leaf_records)
    const int32_t *m2l_perm;  // [n_ent] entries of each level in M2L target order (build_m2l_order)
    const int32_t *m2l_src8;  // [n_ent][8] V-list source entry of a split entry per direction, -1: none
    const double *taylor;  // Laplace L2P coefficients map, or null
    const double *leaf_coef;  // [leaf_list index][2p+1] Taylor coefficients of the leaves (mixed form)
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

// The near-field sources of leaf g: the leaf itself first, then its
// colleagues in direction order, as one list; rng[0..9) is the first list
// position of each range, rng[9..18) the point index minus the list position.
__device__ __forceinline__ int leaf_ranges(const PassArgs &A, int g, int *rng) {
    int ns = 0;
    for (int i = 0; i < 9; i++) {
        const int d = i <= 4 ? i - 1 : i;
        const int c = i == 0 ? g : A.ncoll[9 * (size_t)g + d];
        const int rb = c >= 0 ? A.nbot[c] : 0, rn = c >= 0 ? A.ntop[c] - rb : 0;
        rng[i] = ns;
        rng[9 + i] = rb - ns;
        ns += rn;
    }
    return ns;
}
// point index of list position p
__device__ __forceinline__ int range_point(const int *rng, int p) {
    int sv = p + rng[9];
#pragma unroll
    for (int i = 1; i < 9; i++) sv = p >= rng[i] ? p + rng[9 + i] : sv;
    return sv;
}
// Leaf record (one 128-byte row per entry of the leaf list, built with the
// tree): everything a leaf kernel needs before it gathers, in one coalesced
// warp load instead of the chain list -> node -> colleagues -> their ranges.
enum LeafRec : int {
    LR_NODE = 0, LR_LEVEL = 1, LR_BOT = 2, LR_TOP = 3, LR_NSRC = 4, LR_KEY_LO = 5, LR_KEY_HI = 6,
    LR_RNG = 8,  // [LR_RNG, LR_RNG + 18): the leaf_ranges table
    LEAF_REC_WORDS = 32
};
void build_leaf_records(kifmm_plan *P);
void build_m2l_order(kifmm_plan *P);

// FP64 tensor-core MMA (mma.sync m8n8k4 .f64): D = A B + D with fragments
// A[row = lane/4][k = lane%4], B[k = lane%4][n = lane/4],
// D[row = lane/4][n = 2*(lane%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}
// row stride = 4 mod 16 doubles: conflict-free fragment loads
__host__ __device__ constexpr int pad4mod16(int m) { return m + (20 - m % 16) % 16; }
// planned.cu
void launch_planned_p2m(kifmm_plan *P, const PassArgs &A);
void launch_planned_leaf(kifmm_plan *P, const PassArgs &A);
// passes_complex.cu (complex values: FP64 point passes on double2 densities)
void launch_gather_tau_c(kifmm_plan *P);
void launch_p2m_c(kifmm_plan *P, const PassArgs &A);
void run_eval_sources_c(kifmm_plan *P, const PassArgs &A, int check_self);
void run_eval_targets_c(kifmm_plan *P, const PassArgs &A, const double *tx, const double *ty, int64_t n,
                        int check_self, double *pot);
// passes_mixed.cu
void run_passes_mixed(kifmm_plan *P);
void run_eval_sources_mixed(kifmm_plan *P, int check_self);
void run_eval_targets_mixed(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self,
                            double *pot);

}  // namespace kifmm
