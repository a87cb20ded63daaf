// passes_complex.cu -- the point passes of the complex form, FP64.
//
// The reference's complex mode (FMM(..., iscomplex=True), class_fmm.py:174)
// keeps every workspace in complex128 and runs the same passes.  Here a node's
// state is the real image of its complex check potential: Q = 2 Qc doubles,
// [Re u (Qc), Im u (Qc)], and every translation operator is the real image of
// the complex one (operators.cu), so M2M, M2L and L2L are the real FP64
// kernels unchanged.  What touches points is here:
//   P2M  numba_upwards_pass (class_fmm.py:57-71): check potential on the large
//        circle from the node's sources;
//   L2P + P2P  numba_target_local_expansion_evaluation / neighbor_evaluation
//        (class_fmm.py:73-111), at the sources and at separate targets;
//   KF / KA / KAS (class_fmm.py:115-145) for a complex kernel.
// Densities and potentials are double2 (re, im) in HBM.
#include "passes.cuh"

namespace kifmm {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ void cacc(double2 &acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

__global__ void k_gather_tau_c(const double2 *__restrict__ tau, const int32_t *__restrict__ perm, int64_t n,
                               double2 *__restrict__ taus) {
    pdl_trigger();
    pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        taus[i] = tau[perm[i]];
}

__global__ void k_scatter_pot_c(const double2 *__restrict__ pots, const int32_t *__restrict__ perm, int64_t n,
                                double2 *__restrict__ pot) {
    pdl_trigger();
    pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pot[perm[i]] = pots[i];
}

// P2M: one warp per node; lane q (< Qc <= 32) sums over the node's sources,
// staged 32 at a time in shared memory.
constexpr int P2MC_WARPS = 8;
__global__ void __launch_bounds__(32 * P2MC_WARPS) k_p2m_c(PassArgs A, const int32_t *__restrict__ list, int64_t nlist,
                                                            const double2 *__restrict__ taus) {
    __shared__ double sx[P2MC_WARPS][32], sy[P2MC_WARPS][32];
    __shared__ double2 st[P2MC_WARPS][32];
    pdl_trigger();
    pdl_wait();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, Qc = A.Qc;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= nlist) return;
    const int g = list[w], l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const double *lg = A.ops + (size_t)l * A.stride + A.off_large;  // x [0, Qc), y [Qc, 2 Qc)
    const int b = A.nbot[g], e = A.ntop[g];
    const bool ok = lane < Qc;
    const double tx = ok ? lg[lane] + cx : 0.0, ty = ok ? lg[Qc + lane] + cy : 0.0;
    double2 acc = make_double2(0.0, 0.0);
    for (int s0 = b; s0 < e; s0 += 32) {
        __syncwarp();
        if (s0 + lane < e) {
            sx[wib][lane] = A.xs[s0 + lane];
            sy[wib][lane] = A.ys[s0 + lane];
            st[wib][lane] = taus[s0 + lane];
        }
        __syncwarp();
        const int ns = min(32, e - s0);
        for (int u = 0; u < ns; u++) {
            const double dx = tx - sx[wib][u], dy = ty - sy[wib][u];
            cacc(acc, green_z(A.kind, A.k, dx * dx + dy * dy), st[wib][u]);
        }
    }
    if (ok) {
        A.uup[(size_t)g * A.Q + lane] = acc.x;
        A.uup[(size_t)g * A.Q + Qc + lane] = acc.y;
    }
}

// Local equivalent density of node g (levels >= 2): phi = Inv_l u_down on the
// real image, as (re, im) pairs phi[q], q < Qc.
__device__ __forceinline__ void local_density_c(const PassArgs &A, int g, int l, double *phi) {
    const int Q = A.Q;
    const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
    for (int r = threadIdx.x; r < Q; r += blockDim.x) {
        double s = 0.0;
        if (l >= 2)
            for (int c = 0; c < Q; c++) s = fma(inv[r * Q + c], A.udown[(size_t)g * Q + c], s);
        phi[r] = s;
    }
}

// L2P + P2P for one target leaf per block (class_fmm.py:73-111); the L2P
// evaluates the local density on the large circle in box-relative coordinates
// (class_fmm.py:81-87).
__global__ void k_leaf_eval_c(PassArgs A, const int32_t *__restrict__ list, int check_self,
                              const double2 *__restrict__ taus, double2 *__restrict__ pots) {
    extern __shared__ __align__(16) double smc[];
    const int Q = A.Q, Qc = A.Qc, nb = blockDim.x;
    double *phi = smc;                       // [Q]: Re at [0, Qc), Im at [Qc, Q)
    double2 *st = (double2 *)(smc + Q);      // [nb] (Q even: 16-byte aligned)
    double *sx = (double *)(st + nb), *sy = sx + nb;
    const int g = list[blockIdx.x], l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    local_density_c(A, g, l, phi);
    __syncthreads();
    const double *lg = A.ops + (size_t)l * A.stride + A.off_large;
    const int b = A.nbot[g], e = A.ntop[g];
    for (int t0 = b; t0 < e; t0 += nb) {
        const int t = t0 + threadIdx.x;
        const bool act = t < e;
        const double px = act ? A.xs[t] : 0.0, py = act ? A.ys[t] : 0.0;
        double2 acc = make_double2(0.0, 0.0);
        if (act && l >= 1) {
            const double rx = px - cx, ry = py - cy;
            for (int q = 0; q < Qc; q++) {
                const double dx = rx - lg[q], dy = ry - lg[Qc + q];
                cacc(acc, green_z(A.kind, A.k, dx * dx + dy * dy), make_double2(phi[q], phi[Qc + q]));
            }
        }
        for (int d = 0; d < 9; d++) {
            const int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            const int cb = A.nbot[c], ce = A.ntop[c];
            for (int s0 = cb; s0 < ce; s0 += nb) {
                __syncthreads();
                const int s = s0 + threadIdx.x;
                if (s < ce) {
                    sx[threadIdx.x] = A.xs[s];
                    sy[threadIdx.x] = A.ys[s];
                    st[threadIdx.x] = taus[s];
                }
                __syncthreads();
                const int ns = min(nb, ce - s0);
                if (act)
                    for (int u = 0; u < ns; u++) {
                        const double dx = px - sx[u], dy = py - sy[u];
                        if (check_self && dx == 0.0 && dy == 0.0) continue;
                        cacc(acc, green_z(A.kind, A.k, dx * dx + dy * dy), st[u]);
                    }
            }
        }
        if (act) pots[t] = acc;
    }
}

// separate targets: locate by strict '>' descent (tree.py:712-727), L2P, P2P
__global__ void k_eval_targets_c(PassArgs A, const double *__restrict__ tx, const double *__restrict__ ty, int64_t n,
                                 int check_self, const double2 *__restrict__ taus, double2 *__restrict__ pot) {
    const int Q = A.Q, Qc = A.Qc;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double px = tx[i], py = ty[i];
        int g = 0, l = 0;
        while (A.nflag[g] & NF_SPLIT) {
            double cx, cy;
            node_center(A, g, l, cx, cy);
            g = A.nchild[g] + 2 * (px > cx) + (py > cy);
            l++;
        }
        double cx, cy;
        node_center(A, g, l, cx, cy);
        double2 acc = make_double2(0.0, 0.0);
        if (l >= 2) {
            const double *blk = A.ops + (size_t)l * A.stride;
            const double *inv = blk + A.off_inv, *lg = blk + A.off_large;
            const double *u = A.udown + (size_t)g * Q;
            const double rx = px - cx, ry = py - cy;
            for (int q = 0; q < Qc; q++) {
                double pr = 0.0, pi = 0.0;
                for (int c = 0; c < Q; c++) {
                    pr = fma(inv[q * Q + c], u[c], pr);
                    pi = fma(inv[(Qc + q) * Q + c], u[c], pi);
                }
                const double dx = rx - lg[q], dy = ry - lg[Qc + q];
                cacc(acc, green_z(A.kind, A.k, dx * dx + dy * dy), make_double2(pr, pi));
            }
        }
        for (int d = 0; d < 9; d++) {
            const int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            for (int s = A.nbot[c]; s < A.ntop[c]; s++) {
                const double dx = px - A.xs[s], dy = py - A.ys[s];
                if (check_self && dx == 0.0 && dy == 0.0) continue;
                cacc(acc, green_z(A.kind, A.k, dx * dx + dy * dy), taus[s]);
            }
        }
        pot[i] = acc;
    }
}

// ------------------------------------------------ kernel-function utilities
// KAS restricted to targets (class_fmm.py:134-143), complex: one block per target
__global__ void k_direct_c(int kind, double k, const double *__restrict__ x, const double *__restrict__ y,
                           const double2 *__restrict__ tau, int64_t n, const int64_t *__restrict__ tg,
                           double2 *__restrict__ out) {
    __shared__ double2 red[32];
    const int64_t j = tg[blockIdx.x];
    if (j < 0 || j >= n) {  // caller index out of range: report NaN, touch nothing
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        if (threadIdx.x == 0) out[blockIdx.x] = make_double2(nan, nan);
        return;
    }
    const double px = x[j], py = y[j];
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        if (i == j) continue;
        const double dx = px - x[i], dy = py - y[i];
        cacc(acc, green_z(kind, k, dx * dx + dy * dy), tau[i]);
    }
    for (int o = 16; o; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double2 v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : make_double2(0.0, 0.0);
        for (int o = 16; o; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
        if (threadIdx.x == 0) out[blockIdx.x] = v;
    }
}

__global__ void k_kmatrix_c(int kind, double k, const double *sx, const double *sy, int64_t ns, const double *tx,
                            const double *ty, int64_t nt, double2 *out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ns * nt; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e / ns, i = e % ns;
        const double dx = tx[j] - sx[i], dy = ty[j] - sy[i];
        out[e] = green_z(kind, k, dx * dx + dy * dy);
    }
}

__global__ void k_kapply_c(int kind, double k, const double *sx, const double *sy, int64_t ns, const double *tx,
                           const double *ty, int64_t nt, const double2 *tau, double2 *out) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nt; j += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t i = 0; i < ns; i++) {
            const double dx = tx[j] - sx[i], dy = ty[j] - sy[i];
            cacc(acc, green_z(kind, k, dx * dx + dy * dy), tau[i]);
        }
        out[j] = acc;
    }
}

// ------------------------------------------------------------ host side
void launch_gather_tau_c(kifmm_plan *P) {
    launch_pdl(k_gather_tau_c, dim3(grid_for(P->N, 256, P->num_sms * 8)), dim3(256), 0, P->stream,
               (const double2 *)P->tau.p, (const int32_t *)P->perm.p, P->N, (double2 *)P->taus.p);
}

void launch_p2m_c(kifmm_plan *P, const PassArgs &A) {
    KIFMM_REQUIRE(P->Qc <= 32, KIFMM_ERR_ARG, "complex form: Nequiv above 32");
    launch_pdl(k_p2m_c, dim3(grid_for(P->n_p2m_list * 32, 32 * P2MC_WARPS)), dim3(32 * P2MC_WARPS), 0, P->stream, A,
               (const int32_t *)P->p2m_list.p, P->n_p2m_list, (const double2 *)P->taus.p);
}

void run_eval_sources_c(kifmm_plan *P, const PassArgs &A, int check_self) {
    if (P->n_leaf_list) {
        PhaseScope ph(P, KIFMM_PHASE_LEAF);
        const int thr = P->ppl <= 64 ? 64 : 128;
        const size_t smem = (size_t)(P->Q + 4 * thr) * sizeof(double);
        k_leaf_eval_c<<<(unsigned)P->n_leaf_list, thr, smem, P->stream>>>(A, P->leaf_list.p, check_self,
                                                                           (const double2 *)P->taus.p,
                                                                           (double2 *)P->pots.p);
        KIFMM_LAUNCHED();
    }
    launch_pdl(k_scatter_pot_c, dim3(grid_for(P->N, 256, P->num_sms * 8)), dim3(256), 0, P->stream,
               (const double2 *)P->pots.p, (const int32_t *)P->perm.p, P->N, (double2 *)P->pot_out.p);
}

void run_eval_targets_c(kifmm_plan *P, const PassArgs &A, const double *tx, const double *ty, int64_t n,
                        int check_self, double *pot) {
    k_eval_targets_c<<<grid_for(n, 128, P->num_sms * 16), 128, 0, P->stream>>>(
        A, tx, ty, n, check_self, (const double2 *)P->taus.p, (double2 *)pot);
    KIFMM_LAUNCHED();
}

void direct_sum_device_c(const kifmm_kernel &kn, const double *x, const double *y, const double *tau, int64_t n,
                         const int64_t *tg, int64_t nt, double *out, cudaStream_t s) {
    if (nt <= 0) return;
    KIFMM_REQUIRE(nt < (1ll << 31), KIFMM_ERR_ARG, "direct_sum: too many targets");
    k_direct_c<<<(unsigned)nt, 256, 0, s>>>(kn.kind, kn.k, x, y, (const double2 *)tau, n, tg, (double2 *)out);
    KIFMM_LAUNCHED();
}

void kernel_matrix_device_c(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                            const double *ty, int64_t nt, double *out, cudaStream_t s) {
    if (ns * nt <= 0) return;
    k_kmatrix_c<<<grid_for(ns * nt, 256, 8192), 256, 0, s>>>(kn.kind, kn.k, sx, sy, ns, tx, ty, nt, (double2 *)out);
    KIFMM_LAUNCHED();
}

void kernel_apply_device_c(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                           const double *ty, int64_t nt, const double *tau, double *out, cudaStream_t s) {
    if (nt <= 0) return;
    k_kapply_c<<<grid_for(nt, 128, 8192), 128, 0, s>>>(kn.kind, kn.k, sx, sy, ns, tx, ty, nt, (const double2 *)tau,
                                                        (double2 *)out);
    KIFMM_LAUNCHED();
}

}  // namespace kifmm
