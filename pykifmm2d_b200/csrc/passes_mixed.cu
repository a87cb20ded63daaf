// passes_mixed.cu -- mixed-precision passes.
//
// Same algorithm as passes.cu (reference class_fmm.py:299-399) with
//   * P2P in FP32 on coordinates relative to the box centre (FP64
//     subtraction, then rounding: nearby points keep their relative precision
//     wherever the box sits, as the reference's L2P does with tx = x - xmid,
//     class_fmm.py:81-82);
//   * P2M and L2P in FP64: their terms are weighted by equivalent densities
//     of alternating sign, and FP32 logs there cost ~1.6e-7 each at 1M points
//     (measured), while they are only Q evaluations per point;
//   * check potentials u_up / u_down kept in FP64, M2M and L2L in FP64 (a few
//     percent of the work);
//   * M2L on the tensor cores (m2l_tc.cu): int8 slices with exact int32
//     accumulation (default), or bf16 / fp16 hi-lo splits with FP32
//     accumulation; or FP32 tiles on the CUDA cores (this file);
//   * the local expansion's equivalent density Inv_l u_down formed in FP64.
// Coincident source/target pairs (r^2 == 0 after rounding) contribute zero.
#include "passes.cuh"

namespace kifmm {

constexpr float LN2_OVER_4PI = 0.05515890934390497f;   // ln 2 / (4 pi)
constexpr float INV_2PI_F = 0.15915494309189535f;

// Kernel value in FP32 for relative offsets; Laplace returns log2(r^2)
// (scaled by -ln2/(4pi) once at the end of each sum).
template <int KIND>
__device__ __forceinline__ float gsum_term(float r2, float k) {
    if (KIND == KIFMM_KERNEL_LAPLACE) return __log2f(r2);
    return k0_f(k * sqrtf(r2));
}
template <int KIND>
__device__ __forceinline__ float gsum_scale() {
    return KIND == KIFMM_KERNEL_LAPLACE ? -LN2_OVER_4PI : INV_2PI_F;
}

// Compensated FP32 accumulation (Kahan): sum += term with the lost low part
// carried in c.
struct Kahan {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float term) {
        float y = term - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ void fma_add(float a, float b) {
        float y = fmaf(a, b, -c);
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// FP32 M2L + L2L on the CUDA cores (FP64 state in and out): block = 4Q rows x
// TE target groups.
constexpr int M2LF_TE = 32;
__global__ void k_m2l_f(PassArgs A, int l) {
    extern __shared__ float smf[];
    const int Q = A.Q, Q4 = 4 * Q, r = threadIdx.x;
    float *src = smf;  // [TE][4Q]
    __shared__ int64_t sgrp[M2LF_TE];
    __shared__ int spar[M2LF_TE];
    __shared__ int64_t schild[M2LF_TE];
    const int64_t e0 = (int64_t)blockIdx.x * M2LF_TE;
    const int64_t ne = A.T.ne[l];
    if (r < M2LF_TE) {
        int64_t e = e0 + r;
        bool act = e < ne && !(A.ent[A.T.eoff[l] + e] & 1);
        spar[r] = act ? A.ent_node[A.T.eoff[l] + e] : -1;
        schild[r] = act ? A.T.off[l + 1] + 4 * e : -1;
    }
    __syncthreads();
    float acc[M2LF_TE];
#pragma unroll
    for (int t = 0; t < M2LF_TE; t++) acc[t] = 0.f;
    const float *opl = A.ops_f + (size_t)(l + 1) * A.stride + A.off_m2l;
    for (int d = 0; d < 9; d++) {
        if (d == 4) continue;
        if (r < M2LF_TE) {
            int p = spar[r];
            int64_t grp = -1;
            if (p >= 0) {
                int nb = A.ncoll[9 * (size_t)p + d];
                if (nb >= 0) {
                    int je = A.nent[nb];
                    if (je >= 0) grp = A.T.off[l + 1] + 4 * (je - A.T.eoff[l]);
                }
            }
            sgrp[r] = grp;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < M2LF_TE * Q4; idx += blockDim.x) {
            int t = idx / Q4, c = idx % Q4;
            int64_t grp = sgrp[t];
            src[idx] = grp >= 0 ? (float)A.uup[(size_t)grp * Q + c] : 0.f;
        }
        __syncthreads();
        const float *op = opl + (size_t)d * Q4 * Q4;
        if (r < Q4)
            for (int c = 0; c < Q4; c++) {
                float a = op[(size_t)c * Q4 + r];
#pragma unroll
                for (int t = 0; t < M2LF_TE; t++) acc[t] = fmaf(a, src[t * Q4 + c], acc[t]);
            }
        __syncthreads();
    }
    if (l >= 2) {
        for (int idx = threadIdx.x; idx < M2LF_TE * Q; idx += blockDim.x) {
            int t = idx / Q, c = idx % Q;
            int p = spar[t];
            src[idx] = p >= 0 ? (float)A.udown[(size_t)p * Q + c] : 0.f;
        }
        __syncthreads();
        const float *op = A.ops_f + (size_t)l * A.stride + A.off_l2l;
        if (r < Q4)
            for (int c = 0; c < Q; c++) {
                float a = op[(size_t)c * Q4 + r];
#pragma unroll
                for (int t = 0; t < M2LF_TE; t++) acc[t] = fmaf(a, src[t * Q + c], acc[t]);
            }
    }
    if (r < Q4)
#pragma unroll
        for (int t = 0; t < M2LF_TE; t++)
            if (schild[t] >= 0) A.udown[(size_t)schild[t] * Q + r] = (double)acc[t];
}

// Equivalent density of the local expansion (FP64), for the leaves a warp
// evaluates.
__device__ __forceinline__ void local_density(const PassArgs &A, int g, int l, double *qd, int lane) {
    const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
    for (int r = lane; r < A.Q; r += 32) {
        double s = 0.0;
        if (l >= 2)
            for (int c = 0; c < A.Q; c++) s = fma(inv[r * A.Q + c], A.udown[(size_t)g * A.Q + c], s);
        qd[r] = s;
    }
}

// L2P + P2P: one warp per target leaf, lane per target, 32-source tiles in
// shared memory.  For the Laplace kernel the offsets are scaled by 1/w (w the
// leaf width) so every log2 term is O(1); the remainder log2(w^2) * sum(tau)
// is added in FP64 from per-tile FP64 charge sums (coincident pairs, skipped,
// are taken back out).  Sums are Kahan-compensated.
constexpr int LEAF_WARPS = 4;
template <int KIND>
__global__ void __launch_bounds__(32 * LEAF_WARPS) k_leaf_eval_f(PassArgs A, const int32_t *__restrict__ list,
                                                                 int64_t nlist) {
    constexpr int R = 2 * KIFMM_TAYLOR_P + 1;
    __shared__ float4 tile[LEAF_WARPS][32];
    __shared__ double qds[LEAF_WARPS][R > 64 ? R : 64];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t w = (int64_t)blockIdx.x * LEAF_WARPS + wib;
    if (w >= nlist) return;
    const int g = list[w];
    const int l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const bool lap = KIND == KIFMM_KERNEL_LAPLACE;
    const bool taylor = lap && A.taylor != nullptr && l >= 2;
    double *qd = qds[wib];
    const double width = ldexp(A.W, -l);
    const double sc = lap ? 1.0 / width : 1.0;     // coordinate scale
    const double lw = lap ? -2.0 * log2(sc) : 0.0; // log2 of the squared length unit
    if (taylor) {  // Taylor coefficients of the local expansion (FP64)
        const double *T = A.taylor + (size_t)l * A.Q * R;
        const double *u = A.udown + (size_t)g * A.Q;
        for (int r = lane; r < R; r += 32) {
            double s = 0.0;
            for (int c = 0; c < A.Q; c++) s = fma(T[(size_t)c * R + r], u[c], s);
            qd[r] = s;
        }
    } else {
        local_density(A, g, l, qd, lane);
    }
    __syncwarp();
    const float kk = (float)A.k;
    const int b = A.nbot[g], e = A.ntop[g];
    for (int t0 = b; t0 < e; t0 += 32) {
        const int t = t0 + lane;
        const bool act = t < e;
        const double pxd = act ? A.xs[t] - cx : 0.0, pyd = act ? A.ys[t] - cy : 0.0;
        const float tx = (float)(pxd * sc), ty = (float)(pyd * sc);
        // far field (L2P) in FP64
        double far = 0.0;
        if (l >= 2 && act) {
            const double zx = pxd * sc, zy = pyd * sc;
            if (taylor && zx * zx + zy * zy <= 0.5625) {
                double sr = qd[R - 2], si = qd[R - 1];
                for (int j = KIFMM_TAYLOR_P - 1; j >= 1; j--) {
                    double nr = fma(sr, zx, fma(-si, zy, qd[2 * j - 1]));
                    double ni = fma(sr, zy, fma(si, zx, qd[2 * j]));
                    sr = nr;
                    si = ni;
                }
                far = qd[0] + (sr * zx - si * zy);
            } else {
                // direct FP64 sum over the equivalent points (out-of-box targets, K0)
                const double *lgd = A.ops + (size_t)l * A.stride + A.off_large;
                const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
                const double *u = A.udown + (size_t)g * A.Q;
                for (int q = 0; q < A.Q; q++) {
                    double qq = taylor ? 0.0 : qd[q];
                    if (taylor)
                        for (int c = 0; c < A.Q; c++) qq = fma(inv[q * A.Q + c], u[c], qq);
                    double dx = pxd - lgd[q], dy = pyd - lgd[A.Q + q];
                    far = fma(green_d(A.kind, A.k, dx * dx + dy * dy), qq, far);
                }
            }
        }
        double near = 0.0;  // FP64 sum of per-tile FP32 partial sums
        double tsum = 0.0;  // FP64 sum of the sources' charges
        float excl = 0.f;   // charges of the skipped coincident pairs
#pragma unroll 1
        for (int d = 0; d < 9; d++) {
            const int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            const int cb = A.nbot[c], ce = A.ntop[c];
            for (int s0 = cb; s0 < ce; s0 += 32) {
                const int s = s0 + lane;
                __syncwarp();
                double ts = 0.0;
                // a short tile is padded with far, uncharged sources: fixed 32-wide loop
                float4 v = make_float4(1e18f, 1e18f, 0.f, 0.f);
                if (s < ce) {
                    ts = A.taus[s];
                    v = make_float4((float)((A.xs[s] - cx) * sc), (float)((A.ys[s] - cy) * sc), (float)ts, 0.f);
                }
                tile[wib][lane] = v;
                if (lap) {
                    for (int o = 16; o; o >>= 1) ts += __shfl_xor_sync(0xffffffffu, ts, o);
                    tsum += ts;
                }
                __syncwarp();
                float acc = 0.f;
                if (KIND == KIFMM_KERNEL_LAPLACE) {
#pragma unroll 8
                    for (int u = 0; u < 32; u++) {
                        const float4 sv = tile[wib][u];
                        const float dx = tx - sv.x, dy = ty - sv.y;
                        const float r2 = fmaf(dx, dx, dy * dy);
                        const bool z = r2 == 0.f;  // coincident pair: skipped (class_fmm.py:107)
                        acc = fmaf(sv.z, __log2f(z ? 1.f : r2), acc);
                        excl += z ? sv.z : 0.f;
                    }
                } else {
                    const int ns = min(32, ce - s0);
#pragma unroll 1
                    for (int u = 0; u < ns; u++) {
                        const float4 sv = tile[wib][u];
                        const float dx = tx - sv.x, dy = ty - sv.y;
                        const float r2 = fmaf(dx, dx, dy * dy);
                        if (r2 > 0.f) acc = fmaf(sv.z, gsum_term<KIND>(r2, kk), acc);
                    }
                }
                near += (double)acc;
            }
        }
        if (act) {
            double v = near;
            // the skipped pair is almost always the target itself: take its
            // charge in FP64 so that log2(w^2) * (tsum - excl) cancels exactly
            const double tau_t = A.taus[t];
            const double ex = (excl == (float)tau_t) ? tau_t : (double)excl;
            if (lap) v += lw * (tsum - ex);
            A.pots[t] = v * (double)gsum_scale<KIND>() + far;
        }
    }
}

// separate targets: one thread per target
template <int KIND>
__global__ void k_eval_targets_f(PassArgs A, const double *__restrict__ tx, const double *__restrict__ ty, int64_t n,
                                 double *__restrict__ pot) {
    const float kk = (float)A.k;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double px = tx[i], py = ty[i];
        int g = 0, l = 0;
        while (A.nflag[g] & NF_SPLIT) {
            double cx, cy;
            node_center(A, g, l, cx, cy);
            g = A.nchild[g] + 2 * (px > cx) + (py > cy);
            l++;
        }
        double cx, cy;
        node_center(A, g, l, cx, cy);
        const float rx = (float)(px - cx), ry = (float)(py - cy);
        double far = 0.0;  // L2P in FP64
        if (l >= 2) {
            const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
            const double *lgd = A.ops + (size_t)l * A.stride + A.off_large;
            for (int q = 0; q < A.Q; q++) {
                double qd = 0.0;
                for (int c = 0; c < A.Q; c++) qd = fma(inv[q * A.Q + c], A.udown[(size_t)g * A.Q + c], qd);
                double dx = (px - cx) - lgd[q], dy = (py - cy) - lgd[A.Q + q];
                far = fma(green_d(A.kind, A.k, dx * dx + dy * dy), qd, far);
            }
        }
        float acc = 0.f;
        for (int d = 0; d < 9; d++) {
            int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            for (int s = A.nbot[c]; s < A.ntop[c]; s++) {
                float dx = rx - (float)(A.xs[s] - cx), dy = ry - (float)(A.ys[s] - cy);
                float r2 = fmaf(dx, dx, dy * dy);
                if (r2 > 0.f) acc = fmaf((float)A.taus[s], gsum_term<KIND>(r2, kk), acc);
            }
        }
        pot[i] = (double)(acc * gsum_scale<KIND>()) + far;
    }
}

// m2l_tc.cu / passes.cu
void run_m2l_tensor(kifmm_plan *P, const PassArgs &A);
void launch_p2m_d(kifmm_plan *P, const PassArgs &A);
void launch_leaf_eval_d(kifmm_plan *P, const PassArgs &A, int check_self);
void launch_eval_targets_d(kifmm_plan *P, const PassArgs &A, const double *tx, const double *ty, int64_t n,
                           int check_self, double *pot);
void launch_m2m_d(kifmm_plan *P, const PassArgs &A, int l);
void launch_l2l_d(kifmm_plan *P, const PassArgs &A, int l);

void run_passes_mixed(kifmm_plan *P) {
    cudaStream_t s = P->stream;
    const int Q = P->Q, L = P->L;
    int64_t NN = P->n_nodes;
    KIFMM_CUDA(cudaMemsetAsync(P->uup.p, 0, (size_t)NN * Q * sizeof(double), s));
    KIFMM_CUDA(cudaMemsetAsync(P->udown.p, 0, (size_t)NN * Q * sizeof(double), s));
    if (L < 3) return;
    PassArgs A = make_pass_args(P);
    if (P->n_p2m_list) {
        PhaseScope ph(P, KIFMM_PHASE_P2M);
        launch_p2m_d(P, A);
    }
    {
        PhaseScope ph(P, KIFMM_PHASE_M2M);
        for (int l = L - 2; l >= 2; l--)
            if (P->lt.ne[l]) launch_m2m_d(P, A, l);
    }
    const bool simt = P->opt.m2l == KIFMM_M2L_FP32;
    int thr = ((4 * Q + 31) / 32) * 32;
    size_t smem = (size_t)M2LF_TE * 4 * Q * sizeof(float);
    if (simt) {
        PhaseScope ph(P, KIFMM_PHASE_M2L);
        KIFMM_CUDA(cudaFuncSetAttribute(k_m2l_f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        for (int l = 1; l <= L - 2; l++) {
            int64_t ne = P->lt.ne[l];
            if (!ne) continue;
            k_m2l_f<<<(unsigned)((ne + M2LF_TE - 1) / M2LF_TE), thr, smem, s>>>(A, l);
            KIFMM_LAUNCHED();
        }
        return;
    }
    {
        PhaseScope ph(P, KIFMM_PHASE_M2L);
        KIFMM_CUDA(cudaMemsetAsync(P->scal.p + 15, 0, sizeof(unsigned long long), s));
        run_m2l_tensor(P, A);  // all levels at once
    }
    PhaseScope ph(P, KIFMM_PHASE_L2L);
    for (int l = 2; l <= L - 2; l++)
        if (P->lt.ne[l]) launch_l2l_d(P, A, l);
}

void run_eval_sources_mixed(kifmm_plan *P, int check_self) {
    if (!P->n_leaf_list) return;
    PhaseScope ph(P, KIFMM_PHASE_LEAF);
    PassArgs A = make_pass_args(P);
    if (P->opt.near_fp64) {
        launch_leaf_eval_d(P, A, check_self);
        return;
    }  // FP32 form: coincident pairs always contribute zero
    unsigned gr = (unsigned)((P->n_leaf_list + LEAF_WARPS - 1) / LEAF_WARPS);
    if (P->kern.kind == KIFMM_KERNEL_LAPLACE)
        k_leaf_eval_f<KIFMM_KERNEL_LAPLACE><<<gr, 32 * LEAF_WARPS, 0, P->stream>>>(A, P->leaf_list.p, P->n_leaf_list);
    else
        k_leaf_eval_f<KIFMM_KERNEL_MOD_HELMHOLTZ><<<gr, 32 * LEAF_WARPS, 0, P->stream>>>(A, P->leaf_list.p,
                                                                                        P->n_leaf_list);
    KIFMM_LAUNCHED();
}

void run_eval_targets_mixed(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self,
                            double *pot) {
    PassArgs A = make_pass_args(P);
    if (P->opt.near_fp64) {
        launch_eval_targets_d(P, A, tx, ty, n, check_self, pot);
        return;
    }
    unsigned gr = grid_for(n, 128, P->num_sms * 16);
    if (P->kern.kind == KIFMM_KERNEL_LAPLACE)
        k_eval_targets_f<KIFMM_KERNEL_LAPLACE><<<gr, 128, 0, P->stream>>>(A, tx, ty, n, pot);
    else
        k_eval_targets_f<KIFMM_KERNEL_MOD_HELMHOLTZ><<<gr, 128, 0, P->stream>>>(A, tx, ty, n, pot);
    KIFMM_LAUNCHED();
}

}  // namespace kifmm
