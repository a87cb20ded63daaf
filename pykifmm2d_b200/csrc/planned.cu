// planned.cu -- planned applies: P2M, L2P and the near field as matrices in HBM.
//
// The reference's planner (fmm_planner / planned_fmm, pykifmm2d/fmm.py:530-712,
// :741-814) trades memory for time on repeated densities: it builds once the
// sparse matrices of every P2M kernel evaluation ("upwards" matrices, source
// points -> check circle, build_upwards_pass :472-491), every L2P evaluation
// ("downwards" matrices, large circle -> points) and every near-field pair
// (neighbor matrix, build_neighbor_interactions :429-470), and each apply is
// then sparse matrix products.  Here the same three operators are dense
// per-node blocks in HBM, built by the GPU on the first apply after the tree
// and the operators:
//   P2M   [n_src x Q] per P2M node:   u_up(g)[q]  = sum_s P[s][q] tau_s;
//   L2P   [n_t x Q] per leaf (l >= 2), with the check-to-equivalent inverse
//         folded in: far_t = sum_q L[t][q] u_down(g)[q],
//         L[t][q] = sum_c G(large_c -> t) Inv[c][q];
//   near  [n_t x n_s'] per leaf over the concatenated sources of its 3x3
//         colleagues (rows padded with zeros to 16 bytes):
//         near_t = sum_s N[t][s] tau_s, pairs with equal coordinates zero
//         (evaluate_to_points(..., check_self=True), class_fmm.py:105-108).
// Each apply then streams the blocks once: one CTA per leaf stages the leaf's
// concatenated charges in shared memory and each warp reduces whole target
// rows with 16-byte loads (HBM-bound matrix-vector products).  Values are
// computed in FP64; the near blocks are stored in FP32 for the mixed
// precision (no FP32 coordinate differences are involved), in FP64 otherwise.
#include "passes.cuh"

namespace kifmm {

// block sizes of every leaf (near, L2P) and P2M node
// near rows hold n_s values padded to a multiple of vw (16 bytes)
__host__ __device__ __forceinline__ int64_t pad_row(int64_t ns, int vw) { return (ns + vw - 1) / vw * vw; }
__global__ void k_plan_sizes(PassArgs A, const int32_t *__restrict__ leaves, int64_t nleaf,
                             const int32_t *__restrict__ p2m, int64_t np2m, int vw, int64_t *__restrict__ near_sz,
                             int64_t *__restrict__ l2p_sz, int64_t *__restrict__ p2m_sz) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nleaf + np2m;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < nleaf) {
            const int g = leaves[i];
            const int64_t nt = A.ntop[g] - A.nbot[g];
            int64_t ns = 0;
            for (int d = 0; d < 9; d++) {
                const int c = A.ncoll[9 * (size_t)g + d];
                if (c >= 0) ns += A.ntop[c] - A.nbot[c];
            }
            near_sz[i] = nt * pad_row(ns, vw);
            l2p_sz[i] = A.nlev[g] >= 2 ? (int64_t)A.Q * nt : 0;
        } else {
            const int g = p2m[i - nleaf];
            p2m_sz[i - nleaf] = (int64_t)(A.ntop[g] - A.nbot[g]) * A.Q;
        }
    }
}

// exclusive prefix sums of v[0..n) in place, v[n] = total; one block
constexpr int PS_THREADS = 1024;
__global__ void __launch_bounds__(PS_THREADS) k_plan_scan(int64_t *v, int64_t n) {
    __shared__ int64_t part[PS_THREADS];
    const int64_t per = (n + PS_THREADS - 1) / PS_THREADS, b = threadIdx.x * per, e = min(n, b + per);
    int64_t s = 0;
    for (int64_t i = b; i < e; i++) s += v[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t acc = 0;
        for (int i = 0; i < PS_THREADS; i++) {
            const int64_t t = part[i];
            part[i] = acc;
            acc += t;
        }
        v[n] = acc;
    }
    __syncthreads();
    int64_t acc = part[threadIdx.x];
    for (int64_t i = b; i < e; i++) {
        const int64_t t = v[i];
        v[i] = acc;
        acc += t;
    }
}

template <typename T>
__global__ void k_plan_fill_leaf(PassArgs A, const int32_t *__restrict__ leaves, int64_t nleaf,
                                 const int64_t *__restrict__ near_off, const int64_t *__restrict__ l2p_off,
                                 T *__restrict__ near, double *__restrict__ l2p) {
    __shared__ int rng[18];
    __shared__ int s_ns;
    const int64_t i = blockIdx.x;
    if (i >= nleaf) return;
    const int g = leaves[i], l = A.nlev[g], b = A.nbot[g], nt = A.ntop[g] - b, Q = A.Q;
    if (threadIdx.x == 0) s_ns = leaf_ranges(A, g, rng);
    __syncthreads();
    const int ns = s_ns, nsp = (int)((near_off[i + 1] - near_off[i]) / max(nt, 1));
    T *nb = near + near_off[i];
    for (int64_t e = threadIdx.x; e < (int64_t)nt * nsp; e += blockDim.x) {
        const int t = (int)(e / nsp), s = (int)(e % nsp);
        double v = 0.0;
        if (s < ns) {
            const int sp = range_point(rng, s);
            const double dx = A.xs[b + t] - A.xs[sp], dy = A.ys[b + t] - A.ys[sp];
            v = (dx == 0.0 && dy == 0.0) ? 0.0 : green_d(A.kind, A.k, dx * dx + dy * dy);
        }
        nb[e] = (T)v;
    }
    if (l < 2) return;
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const double *blk = A.ops + (size_t)l * A.stride;
    const double *inv = blk + A.off_inv, *lg = blk + A.off_large;
    double *lb = l2p + l2p_off[i];
    for (int e = threadIdx.x; e < nt * Q; e += blockDim.x) {
        const int t = e / Q, q = e % Q;
        const double px = A.xs[b + t] - cx, py = A.ys[b + t] - cy;
        double acc = 0.0;
        for (int c = 0; c < Q; c++) {
            const double dx = px - lg[c], dy = py - lg[Q + c];
            acc = fma(green_d(A.kind, A.k, dx * dx + dy * dy), inv[c * Q + q], acc);
        }
        lb[e] = acc;
    }
}

__global__ void k_plan_fill_p2m(PassArgs A, const int32_t *__restrict__ p2m, int64_t np2m,
                                const int64_t *__restrict__ p2m_off, double *__restrict__ mat) {
    const int64_t i = blockIdx.x;
    if (i >= np2m) return;
    const int g = p2m[i], l = A.nlev[g], b = A.nbot[g], n = A.ntop[g] - b, Q = A.Q;
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const double *lg = A.ops + (size_t)l * A.stride + A.off_large;
    double *m = mat + p2m_off[i];
    for (int e = threadIdx.x; e < n * Q; e += blockDim.x) {
        const int s = e / Q, q = e % Q;
        const double dx = lg[q] + cx - A.xs[b + s], dy = lg[Q + q] + cy - A.ys[b + s];
        m[e] = green_d(A.kind, A.k, dx * dx + dy * dy);
    }
}

// planned P2M: one warp per node, lanes over the Q check points
__global__ void k_planned_p2m(PassArgs A, const int32_t *__restrict__ p2m, int64_t np2m,
                              const int64_t *__restrict__ p2m_off, const double *__restrict__ mat) {
    pdl_trigger();
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= np2m) return;
    const int g = p2m[w], b = A.nbot[g], n = A.ntop[g] - b, Q = A.Q;
    const double *m = mat + p2m_off[w];
    for (int q0 = 0; q0 < Q; q0 += 32) {
        const int q = q0 + lane;
        double acc0 = 0.0, acc1 = 0.0;
        if (q < Q) {
            int s = 0;
            for (; s + 1 < n; s += 2) {
                acc0 = fma(m[(size_t)s * Q + q], A.taus[b + s], acc0);
                acc1 = fma(m[(size_t)(s + 1) * Q + q], A.taus[b + s + 1], acc1);
            }
            if (s < n) acc0 = fma(m[(size_t)s * Q + q], A.taus[b + s], acc0);
            A.uup[(size_t)g * Q + q] = acc0 + acc1;
        }
    }
}

// planned L2P + near field: one CTA per leaf.  The leaf's concatenated
// charges are staged in shared memory (PL_CHUNK at a time), its u_down too;
// each warp takes whole target rows, lanes over the row with 16-byte loads
// (FP32 rows: products summed in FP32 per lane, then in FP64 across lanes).
constexpr int PL_THREADS = 128, PL_CHUNK = 1024;
template <typename T>
__global__ void __launch_bounds__(PL_THREADS) k_planned_leaf(PassArgs A, const int32_t *__restrict__ leaves,
                                                             int64_t nleaf, const int64_t *__restrict__ near_off,
                                                             const int64_t *__restrict__ l2p_off,
                                                             const T *__restrict__ near,
                                                             const double *__restrict__ l2p) {
    constexpr int VW = 16 / sizeof(T);  // values per 16-byte load
    extern __shared__ __align__(16) double pl_sm[];
    T *tch = (T *)pl_sm;                                   // [PL_CHUNK] charges of the chunk
    double *us = pl_sm + PL_CHUNK;                         // [Q] u_down of the leaf
    double *acc = us + A.Q;                                // [n_t] per-target sums
    __shared__ int rng[18];
    __shared__ int s_ns;
    pdl_trigger();
    pdl_wait();
    const int64_t i = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = PL_THREADS / 32;
    const int g = leaves[i], l = A.nlev[g], b = A.nbot[g], nt = A.ntop[g] - b, Q = A.Q;
    if (tid == 0) s_ns = leaf_ranges(A, g, rng);
    for (int q = tid; q < Q; q += PL_THREADS) us[q] = l >= 2 ? A.udown[(size_t)g * Q + q] : 0.0;
    __syncthreads();
    const int ns = s_ns, nsp = (int)((near_off[i + 1] - near_off[i]) / max(nt, 1));
    // far field: L2P rows
    const double *lb = l2p + l2p_off[i];
    for (int t = warp; t < nt; t += nw) {
        double f = 0.0;
        if (l >= 2)
            for (int q = lane; q < Q; q += 32) f = fma(lb[(size_t)t * Q + q], us[q], f);
        for (int o = 16; o; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
        if (lane == 0) acc[t] = f;
    }
    const T *nb = near + near_off[i];
    for (int c0 = 0; c0 < nsp; c0 += PL_CHUNK) {
        const int cn = min(PL_CHUNK, nsp - c0);  // a multiple of VW
        __syncthreads();
        for (int s = tid; s < cn; s += PL_THREADS)
            tch[s] = c0 + s < ns ? (T)A.taus[range_point(rng, c0 + s)] : (T)0;
        __syncthreads();
        for (int t = warp; t < nt; t += nw) {
            const T *row = nb + (size_t)t * nsp + c0;
            T part = 0;
#pragma unroll 2
            for (int s = lane * VW; s < cn; s += 32 * VW) {
                if (VW == 4) {
                    const float4 m = *(const float4 *)(row + s);
                    const float4 v = *(const float4 *)(tch + s);
                    part = fmaf(m.x, v.x, fmaf(m.y, v.y, fmaf(m.z, v.z, fmaf(m.w, v.w, part))));
                } else {
                    const double2 m = *(const double2 *)(row + s);
                    const double2 v = *(const double2 *)(tch + s);
                    part = fma(m.x, v.x, fma(m.y, v.y, part));
                }
            }
            double d = (double)part;
            for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
            if (lane == 0) acc[t] += d;
        }
    }
    __syncthreads();
    for (int t = tid; t < nt; t += PL_THREADS) A.pots[b + t] = acc[t];
}

// ------------------------------------------------------------ host side
bool planned_ready(const kifmm_plan *P) { return P->opt.planned && P->have_mats; }

void build_plan_matrices(kifmm_plan *P) {
    if (!P->opt.planned || P->have_mats) return;
    KIFMM_REQUIRE(!P->cplx, KIFMM_ERR_UNSUPPORTED, "planned applies: real values only");
    cudaStream_t s = P->stream;
    const int64_t nl = P->n_leaf_list, np = P->n_p2m_list;
    PassArgs A = make_pass_args(P);
    P->pm_near_off.alloc(nl + 1);
    P->pm_l2p_off.alloc(nl + 1);
    P->pm_p2m_off.alloc(np + 1);
    KIFMM_CUDA(cudaMemsetAsync(P->pm_near_off.p, 0, (nl + 1) * 8, s));
    KIFMM_CUDA(cudaMemsetAsync(P->pm_l2p_off.p, 0, (nl + 1) * 8, s));
    KIFMM_CUDA(cudaMemsetAsync(P->pm_p2m_off.p, 0, (np + 1) * 8, s));
    if (nl + np) {
        k_plan_sizes<<<grid_for(nl + np, 256, P->num_sms * 8), 256, 0, s>>>(
            A, P->leaf_list.p, nl, P->p2m_list.p, np, P->opt.precision == KIFMM_PREC_MIXED ? 4 : 2,
            P->pm_near_off.p, P->pm_l2p_off.p, P->pm_p2m_off.p);
        KIFMM_LAUNCHED();
    }
    int64_t tot[3];
    int64_t *offs[3] = {P->pm_near_off.p, P->pm_l2p_off.p, P->pm_p2m_off.p};
    const int64_t cnt[3] = {nl, nl, np};
    for (int k = 0; k < 3; k++) {
        k_plan_scan<<<1, PS_THREADS, 0, s>>>(offs[k], cnt[k]);
        KIFMM_LAUNCHED();
        KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_STATS + k, offs[k] + cnt[k], 8, cudaMemcpyDeviceToHost, s));
    }
    KIFMM_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < 3; k++) tot[k] = (int64_t)P->hpin[HP_STATS + k];
    const bool f32 = P->opt.precision == KIFMM_PREC_MIXED;
    if (f32) P->pm_near32.alloc(tot[0]);
    else P->pm_near64.alloc(tot[0]);
    P->pm_l2p.alloc(tot[1]);
    P->pm_p2m.alloc(tot[2]);
    if (nl) {
        if (f32)
            k_plan_fill_leaf<float><<<(unsigned)nl, 256, 0, s>>>(A, P->leaf_list.p, nl, P->pm_near_off.p,
                                                                  P->pm_l2p_off.p, P->pm_near32.p, P->pm_l2p.p);
        else
            k_plan_fill_leaf<double><<<(unsigned)nl, 256, 0, s>>>(A, P->leaf_list.p, nl, P->pm_near_off.p,
                                                                   P->pm_l2p_off.p, P->pm_near64.p, P->pm_l2p.p);
        KIFMM_LAUNCHED();
    }
    if (np) {
        k_plan_fill_p2m<<<(unsigned)np, 256, 0, s>>>(A, P->p2m_list.p, np, P->pm_p2m_off.p, P->pm_p2m.p);
        KIFMM_LAUNCHED();
    }
    P->pm_bytes = (size_t)tot[0] * (f32 ? 4 : 8) + (size_t)(tot[1] + tot[2]) * 8;
    P->have_mats = true;
}

void launch_planned_p2m(kifmm_plan *P, const PassArgs &A) {
    launch_pdl(k_planned_p2m, dim3(grid_for(P->n_p2m_list * 32, 256)), dim3(256), 0, P->stream, A,
               (const int32_t *)P->p2m_list.p, P->n_p2m_list, (const int64_t *)P->pm_p2m_off.p,
               (const double *)P->pm_p2m.p);
}

void launch_planned_leaf(kifmm_plan *P, const PassArgs &A) {
    const dim3 grid((unsigned)P->n_leaf_list), block(PL_THREADS);
    const size_t smem = (size_t)(PL_CHUNK + P->Q + P->ppl) * sizeof(double);  // leaves hold <= Ncutoff points
    if (P->opt.precision == KIFMM_PREC_MIXED) {
        ensure_dyn_smem(k_planned_leaf<float>, smem);
        launch_pdl(k_planned_leaf<float>, grid, block, smem, P->stream, A, (const int32_t *)P->leaf_list.p,
                   P->n_leaf_list, (const int64_t *)P->pm_near_off.p, (const int64_t *)P->pm_l2p_off.p,
                   (const float *)P->pm_near32.p, (const double *)P->pm_l2p.p);
    } else {
        ensure_dyn_smem(k_planned_leaf<double>, smem);
        launch_pdl(k_planned_leaf<double>, grid, block, smem, P->stream, A, (const int32_t *)P->leaf_list.p,
                   P->n_leaf_list, (const int64_t *)P->pm_near_off.p, (const int64_t *)P->pm_l2p_off.p,
                   (const double *)P->pm_near64.p, (const double *)P->pm_l2p.p);
    }
}

}  // namespace kifmm
