// passes_mixed.cu -- mixed-precision passes.
//
// Same algorithm as passes.cu (reference class_fmm.py:299-399) with
//   * P2M, L2P and P2P in FP32 on coordinates relative to the box centre
//     (FP64 subtraction, then rounding: nearby points keep their relative
//     precision wherever the box sits, as the reference's L2P does with
//     tx = x - xmid, class_fmm.py:81-82);
//   * check potentials u_up / u_down stored in FP32;
//   * M2M, L2L and M2L applied with FP32 operators (the FP64 operators of
//     operators.cu rounded once), M2L either on the CUDA cores (this file) or
//     on the tensor cores with compensated half-precision splits (m2l_tc.cu);
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

template <int KIND>
__global__ void k_p2m_f(PassArgs A, const int32_t *__restrict__ list, int64_t nlist) {
    const int lane = threadIdx.x & 31;
    int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= nlist) return;
    int g = list[w];
    int l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const bool lap = KIND == KIFMM_KERNEL_LAPLACE;
    const double sc = lap ? 1.0 / ldexp(A.W, -l) : 1.0;
    const double lw = lap ? -2.0 * log2(sc) : 0.0;
    const float fsc = (float)sc;
    const float *lg = A.ops_f + (size_t)l * A.stride + A.off_large;
    const float kk = (float)A.k;
    const int b = A.nbot[g], e = A.ntop[g];
    for (int q0 = 0; q0 < A.Q; q0 += 32) {
        int q = q0 + lane;
        bool ok = q < A.Q;
        float tx = ok ? lg[q] * fsc : 0.f, ty = ok ? lg[A.Q + q] * fsc : 0.f;
        Kahan acc;
        double tsum = 0.0;
        for (int s = b; s < e; s++) {
            float dx = tx - (float)((A.xs[s] - cx) * sc), dy = ty - (float)((A.ys[s] - cy) * sc);
            float r2 = fmaf(dx, dx, dy * dy);
            acc.fma_add((float)A.taus[s], gsum_term<KIND>(r2, kk));
            tsum += A.taus[s];
        }
        double v = acc.value() + (lap ? lw * tsum : 0.0);
        if (ok) A.uup_f[(size_t)g * A.Q + q] = (float)(v * (double)gsum_scale<KIND>());
    }
}

__global__ void k_m2m_f(PassArgs A, int l) {
    extern __shared__ float svf[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int Q = A.Q, Q4 = 4 * Q;
    float *v = svf + (size_t)wib * Q4;
    bool active = e < A.T.ne[l];
    int64_t j = A.T.eoff[l] + e;
    int64_t c0 = active ? A.T.off[l + 1] + 4 * e : 0;
    if (active)
        for (int c = lane; c < Q4; c += 32) v[c] = A.uup_f[(size_t)c0 * Q + c];
    __syncwarp();
    if (!active) return;
    int g = A.ent_node[j];
    const float *op = A.ops_f + (size_t)l * A.stride + A.off_m2m;
    for (int r = lane; r < Q; r += 32) {
        float acc = 0.f;
        for (int c = 0; c < Q4; c++) acc = fmaf(op[(size_t)c * Q + r], v[c], acc);
        A.uup_f[(size_t)g * Q + r] = acc;
    }
}

// FP32 M2L + L2L on the CUDA cores: block = 4Q rows x TE target groups.
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
            src[idx] = grp >= 0 ? A.uup_f[(size_t)grp * Q + c] : 0.f;
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
            src[idx] = p >= 0 ? A.udown_f[(size_t)p * Q + c] : 0.f;
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
            if (schild[t] >= 0) A.udown_f[(size_t)schild[t] * Q + r] = acc[t];
}

// L2L alone (used next to the tensor-core M2L): u_down(children) += L2L u_down(parent).
__global__ void k_l2l_f(PassArgs A, int l) {
    extern __shared__ float svl[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int Q = A.Q, Q4 = 4 * Q;
    float *v = svl + (size_t)wib * Q;
    bool active = e < A.T.ne[l] && !(A.ent[A.T.eoff[l] + e] & 1);
    int p = active ? A.ent_node[A.T.eoff[l] + e] : 0;
    if (active)
        for (int c = lane; c < Q; c += 32) v[c] = A.udown_f[(size_t)p * Q + c];
    __syncwarp();
    if (!active) return;
    int64_t c0 = A.T.off[l + 1] + 4 * e;
    const float *op = A.ops_f + (size_t)l * A.stride + A.off_l2l;
    for (int r = lane; r < Q4; r += 32) {
        float acc = 0.f;
        for (int c = 0; c < Q; c++) acc = fmaf(op[(size_t)c * Q4 + r], v[c], acc);
        A.udown_f[(size_t)c0 * Q + r] += acc;
    }
}

// Equivalent density of the local expansion, FP64 product of the FP32 check
// potential, for the leaves a warp evaluates.
__device__ __forceinline__ void local_density(const PassArgs &A, int g, int l, float *qd, int lane) {
    const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
    for (int r = lane; r < A.Q; r += 32) {
        double s = 0.0;
        if (l >= 2)
            for (int c = 0; c < A.Q; c++) s = fma(inv[r * A.Q + c], (double)A.udown_f[(size_t)g * A.Q + c], s);
        qd[r] = (float)s;
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
    __shared__ float4 tile[LEAF_WARPS][32];
    __shared__ float qds[LEAF_WARPS][64];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t w = (int64_t)blockIdx.x * LEAF_WARPS + wib;
    if (w >= nlist) return;
    const int g = list[w];
    const int l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    float *qd = qds[wib];
    local_density(A, g, l, qd, lane);
    __syncwarp();
    const bool lap = KIND == KIFMM_KERNEL_LAPLACE;
    const double width = ldexp(A.W, -l);
    const double sc = lap ? 1.0 / width : 1.0;     // coordinate scale
    const double lw = lap ? -2.0 * log2(sc) : 0.0; // log2 of the squared length unit
    const float kk = (float)A.k;
    const float fsc = (float)sc;
    const float *lg = A.ops_f + (size_t)l * A.stride + A.off_large;
    const int b = A.nbot[g], e = A.ntop[g];
    int coll[9];
#pragma unroll
    for (int d = 0; d < 9; d++) coll[d] = A.ncoll[9 * (size_t)g + d];
    for (int t0 = b; t0 < e; t0 += 32) {
        const int t = t0 + lane;
        const bool act = t < e;
        const float tx = act ? (float)((A.xs[t] - cx) * sc) : 0.f, ty = act ? (float)((A.ys[t] - cy) * sc) : 0.f;
        // far field: equivalent density on the (scaled) check circle
        Kahan far;
        double qsum = 0.0;
        if (l >= 2) {
            for (int q = 0; q < A.Q; q++) {
                float dx = tx - lg[q] * fsc, dy = ty - lg[A.Q + q] * fsc;
                far.fma_add(qd[q], gsum_term<KIND>(fmaf(dx, dx, dy * dy), kk));
                qsum += (double)qd[q];
            }
        }
        Kahan near;
        double tsum = 0.0;  // FP64 sum of the sources' charges
        float excl = 0.f;   // charges of the skipped coincident pairs
#pragma unroll 1
        for (int d = 0; d < 9; d++) {
            const int c = coll[d];
            if (c < 0) continue;
            const int cb = A.nbot[c], ce = A.ntop[c];
            for (int s0 = cb; s0 < ce; s0 += 32) {
                const int s = s0 + lane;
                __syncwarp();
                double ts = 0.0;
                if (s < ce) {
                    ts = A.taus[s];
                    tile[wib][lane] = make_float4((float)((A.xs[s] - cx) * sc), (float)((A.ys[s] - cy) * sc),
                                                  (float)ts, 0.f);
                }
                if (lap) {
                    for (int o = 16; o; o >>= 1) ts += __shfl_xor_sync(0xffffffffu, ts, o);
                    tsum += ts;
                }
                __syncwarp();
                const int ns = min(32, ce - s0);
#pragma unroll 8
                for (int u = 0; u < ns; u++) {
                    const float4 sv = tile[wib][u];
                    const float dx = tx - sv.x, dy = ty - sv.y;
                    const float r2 = fmaf(dx, dx, dy * dy);
                    float gv = 0.f;
                    if (r2 > 0.f) gv = gsum_term<KIND>(r2, kk);
                    else excl += sv.z;
                    near.fma_add(sv.z, gv);
                }
            }
        }
        if (act) {
            double v = far.value() + near.value();
            if (lap) v += lw * (qsum + tsum - (double)excl);
            A.pots[t] = v * (double)gsum_scale<KIND>();
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
        float acc = 0.f;
        if (l >= 2) {
            const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
            const float *lg = A.ops_f + (size_t)l * A.stride + A.off_large;
            for (int q = 0; q < A.Q; q++) {
                double qd = 0.0;
                for (int c = 0; c < A.Q; c++) qd = fma(inv[q * A.Q + c], (double)A.udown_f[(size_t)g * A.Q + c], qd);
                float dx = rx - lg[q], dy = ry - lg[A.Q + q];
                acc = fmaf((float)qd, gsum_term<KIND>(fmaf(dx, dx, dy * dy), kk), acc);
            }
        }
        for (int d = 0; d < 9; d++) {
            int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            for (int s = A.nbot[c]; s < A.ntop[c]; s++) {
                float dx = rx - (float)(A.xs[s] - cx), dy = ry - (float)(A.ys[s] - cy);
                float r2 = fmaf(dx, dx, dy * dy);
                if (r2 > 0.f) acc = fmaf((float)A.taus[s], gsum_term<KIND>(r2, kk), acc);
            }
        }
        pot[i] = (double)(acc * gsum_scale<KIND>());
    }
}

// tensor-core M2L (m2l_tc.cu); returns false when the form is unavailable
bool run_m2l_tensor(kifmm_plan *P, const PassArgs &A, int l);

void run_passes_mixed(kifmm_plan *P) {
    cudaStream_t s = P->stream;
    const int Q = P->Q, L = P->L;
    int64_t NN = P->n_nodes;
    P->uup_f.alloc((size_t)NN * Q);
    P->udown_f.alloc((size_t)NN * Q);
    KIFMM_CUDA(cudaMemsetAsync(P->uup_f.p, 0, (size_t)NN * Q * sizeof(float), s));
    KIFMM_CUDA(cudaMemsetAsync(P->udown_f.p, 0, (size_t)NN * Q * sizeof(float), s));
    if (L < 3) return;
    PassArgs A = make_pass_args(P);
    if (P->n_p2m_list) {
        PhaseScope ph(P, KIFMM_PHASE_P2M);
        unsigned gr = grid_for(P->n_p2m_list * 32, 256);
        if (P->kern.kind == KIFMM_KERNEL_LAPLACE) k_p2m_f<KIFMM_KERNEL_LAPLACE><<<gr, 256, 0, s>>>(A, P->p2m_list.p, P->n_p2m_list);
        else k_p2m_f<KIFMM_KERNEL_MOD_HELMHOLTZ><<<gr, 256, 0, s>>>(A, P->p2m_list.p, P->n_p2m_list);
        KIFMM_LAUNCHED();
    }
    {
        PhaseScope ph(P, KIFMM_PHASE_M2M);
        for (int l = L - 2; l >= 2; l--) {
            int64_t ne = P->lt.ne[l];
            if (!ne) continue;
            k_m2m_f<<<grid_for(ne * 32, 256), 256, (size_t)8 * 4 * Q * sizeof(float), s>>>(A, l);
            KIFMM_LAUNCHED();
        }
    }
    PhaseScope ph(P, KIFMM_PHASE_M2L);
    int thr = ((4 * Q + 31) / 32) * 32;
    size_t smem = (size_t)M2LF_TE * 4 * Q * sizeof(float);
    KIFMM_CUDA(cudaFuncSetAttribute(k_m2l_f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int l = 1; l <= L - 2; l++) {
        int64_t ne = P->lt.ne[l];
        if (!ne) continue;
        bool tc = (P->opt.m2l == KIFMM_M2L_BF16X3 || P->opt.m2l == KIFMM_M2L_FP16X3) && run_m2l_tensor(P, A, l);
        if (tc) {
            if (l >= 2) {
                k_l2l_f<<<grid_for(ne * 32, 256), 256, (size_t)8 * Q * sizeof(float), s>>>(A, l);
                KIFMM_LAUNCHED();
            }
        } else {
            k_m2l_f<<<(unsigned)((ne + M2LF_TE - 1) / M2LF_TE), thr, smem, s>>>(A, l);
            KIFMM_LAUNCHED();
        }
    }
}

void run_eval_sources_mixed(kifmm_plan *P, int check_self) {
    (void)check_self;  // coincident pairs always contribute zero in this form
    if (!P->n_leaf_list) return;
    PhaseScope ph(P, KIFMM_PHASE_LEAF);
    PassArgs A = make_pass_args(P);
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
    (void)check_self;
    PassArgs A = make_pass_args(P);
    unsigned gr = grid_for(n, 128, P->num_sms * 16);
    if (P->kern.kind == KIFMM_KERNEL_LAPLACE)
        k_eval_targets_f<KIFMM_KERNEL_LAPLACE><<<gr, 128, 0, P->stream>>>(A, tx, ty, n, pot);
    else
        k_eval_targets_f<KIFMM_KERNEL_MOD_HELMHOLTZ><<<gr, 128, 0, P->stream>>>(A, tx, ty, n, pot);
    KIFMM_LAUNCHED();
}

}  // namespace kifmm
