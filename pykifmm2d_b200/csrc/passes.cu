// passes.cu -- FMM passes in FP64 (the "plain" form) and their drivers.
//
// Reference: FMM.build_expansions (pykifmm2d/class_fmm.py:299-352) and
// FMM.evaluate_to_points (:379-399).  State is kept as check potentials:
//   u_up   (reference Check_Us)        -- upward check potential of a node;
//   u_down (reference Local_Solutions) -- downward check potential of a node.
// Nodes of a level are stored sibling-group contiguous, so the four children
// of an entry (split or X-list cell) form one 4Q vector.
#include "kifmm_internal.cuh"
#include "passes.cuh"

namespace kifmm {

__global__ void k_gather_tau(const double *__restrict__ tau, const int32_t *__restrict__ perm, int64_t n,
                             double *__restrict__ taus) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        taus[i] = tau[perm[i]];
}

__global__ void k_scatter_pot(const double *__restrict__ pots, const int32_t *__restrict__ perm, int64_t n,
                              double *__restrict__ pot) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pot[perm[i]] = pots[i];
}

// P2M (numba_upwards_pass, class_fmm.py:57-71): one warp per node; lane q
// accumulates over the node's sources in order.
__global__ void k_p2m_d(PassArgs A, const int32_t *__restrict__ list, int64_t nlist) {
    const int lane = threadIdx.x & 31;
    int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= nlist) return;
    int g = list[w];
    int l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const double *lg = A.ops + (size_t)l * A.stride + A.off_large;
    for (int q0 = 0; q0 < A.Q; q0 += 32) {
        int q = q0 + lane;
        bool ok = q < A.Q;
        double tx = ok ? lg[q] + cx : 0.0, ty = ok ? lg[A.Q + q] + cy : 0.0;
        double acc = 0.0;
        for (int s = A.nbot[g]; s < A.ntop[g]; s++) {
            double dx = tx - A.xs[s], dy = ty - A.ys[s];
            acc += green_d(A.kind, A.k, dx * dx + dy * dy) * A.taus[s];
        }
        if (ok) A.uup[(size_t)g * A.Q + q] = acc;
    }
}

// M2M for the entries (split or X-list cells) of level l: one warp each.
__global__ void k_m2m_d(PassArgs A, int l) {
    extern __shared__ double sv[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int Q = A.Q, Q4 = 4 * Q;
    double *v = sv + (size_t)wib * Q4;
    bool active = e < A.T.ne[l];
    int64_t j = A.T.eoff[l] + e;
    int64_t c0 = active ? A.T.off[l + 1] + 4 * e : 0;
    if (active)
        for (int c = lane; c < Q4; c += 32) v[c] = A.uup[(size_t)c0 * Q + c];
    __syncwarp();
    if (!active) return;
    int g = A.ent_node[j];
    const double *op = A.ops + (size_t)l * A.stride + A.off_m2m;  // [4Q][Q]
    for (int r = lane; r < Q; r += 32) {
        double acc = 0.0;
        for (int c = 0; c < Q4; c++) acc = fma(op[(size_t)c * Q + r], v[c], acc);
        A.uup[(size_t)g * Q + r] = acc;
    }
}

// M2L + L2L into the children of the split entries of level l (targets on
// level l+1): class_fmm.py:324-343.  A block owns M2L_TE entries and 4Q rows;
// for each parent direction the source groups are staged in shared memory
// and the column-major operator is streamed once per block.
constexpr int M2L_TE = 16;
__global__ void k_m2l_d(PassArgs A, int l) {
    extern __shared__ double sm[];
    const int Q = A.Q, Q4 = 4 * Q, r = threadIdx.x;
    double *src = sm;                         // [TE][4Q]
    __shared__ int64_t sgrp[M2L_TE];
    __shared__ int spar[M2L_TE];
    __shared__ int64_t schild[M2L_TE];
    const int64_t e0 = (int64_t)blockIdx.x * M2L_TE;
    const int64_t ne = A.T.ne[l];
    if (r < M2L_TE) {
        int64_t e = e0 + r;
        bool act = e < ne && !(A.ent[A.T.eoff[l] + e] & 1);
        spar[r] = act ? A.ent_node[A.T.eoff[l] + e] : -1;
        schild[r] = act ? A.T.off[l + 1] + 4 * e : -1;
    }
    __syncthreads();
    double acc[M2L_TE];
#pragma unroll
    for (int t = 0; t < M2L_TE; t++) acc[t] = 0.0;
    const double *opl = A.ops + (size_t)(l + 1) * A.stride + A.off_m2l;
    for (int d = 0; d < 9; d++) {
        if (d == 4) continue;
        if (r < M2L_TE) {
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
        for (int idx = threadIdx.x; idx < M2L_TE * Q4; idx += blockDim.x) {
            int t = idx / Q4, c = idx % Q4;
            int64_t grp = sgrp[t];
            src[idx] = grp >= 0 ? A.uup[(size_t)grp * Q + c] : 0.0;
        }
        __syncthreads();
        const double *op = opl + (size_t)d * Q4 * Q4;
        if (r < Q4)
            for (int c = 0; c < Q4; c++) {
                double a = op[(size_t)c * Q4 + r];
#pragma unroll
                for (int t = 0; t < M2L_TE; t++) acc[t] = fma(a, src[t * Q4 + c], acc[t]);
            }
        __syncthreads();
    }
    if (l >= 2) {  // L2L from the parents' downward check potentials
        for (int idx = threadIdx.x; idx < M2L_TE * Q; idx += blockDim.x) {
            int t = idx / Q, c = idx % Q;
            int p = spar[t];
            src[idx] = p >= 0 ? A.udown[(size_t)p * Q + c] : 0.0;
        }
        __syncthreads();
        const double *op = A.ops + (size_t)l * A.stride + A.off_l2l;  // [Q][4Q]
        if (r < Q4)
            for (int c = 0; c < Q; c++) {
                double a = op[(size_t)c * Q4 + r];
#pragma unroll
                for (int t = 0; t < M2L_TE; t++) acc[t] = fma(a, src[t * Q + c], acc[t]);
            }
    }
    if (r < Q4)
#pragma unroll
        for (int t = 0; t < M2L_TE; t++)
            if (schild[t] >= 0) A.udown[(size_t)schild[t] * Q + r] = acc[t];
}

// L2P + P2P for one target leaf per block (class_fmm.py:73-111).
__global__ void k_leaf_eval_d(PassArgs A, const int32_t *__restrict__ list, int check_self) {
    extern __shared__ double sm[];
    const int Q = A.Q;
    double *qd = sm;                    // [Q] equivalent density of the local expansion
    double *sx = sm + Q, *sy = sx + blockDim.x, *st = sy + blockDim.x;
    int g = list[blockIdx.x];
    int l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const double *blk = A.ops + (size_t)l * A.stride;
    if (l >= 2) {
        const double *inv = blk + A.off_inv;
        for (int r = threadIdx.x; r < Q; r += blockDim.x) {
            double s = 0.0;
            for (int c = 0; c < Q; c++) s = fma(inv[r * Q + c], A.udown[(size_t)g * Q + c], s);
            qd[r] = s;
        }
    } else {
        for (int r = threadIdx.x; r < Q; r += blockDim.x) qd[r] = 0.0;
    }
    __syncthreads();
    const double *lg = blk + A.off_large;
    const int b = A.nbot[g], e = A.ntop[g];
    for (int t0 = b; t0 < e; t0 += blockDim.x) {
        int t = t0 + threadIdx.x;
        bool act = t < e;
        double px = act ? A.xs[t] : 0.0, py = act ? A.ys[t] : 0.0;
        double acc = 0.0;
        if (act && l >= 1) {
            double tx = px - cx, ty = py - cy;
            for (int q = 0; q < Q; q++) {
                double dx = tx - lg[q], dy = ty - lg[Q + q];
                acc += green_d(A.kind, A.k, dx * dx + dy * dy) * qd[q];
            }
        }
        for (int d = 0; d < 9; d++) {
            int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            int cb = A.nbot[c], ce = A.ntop[c];
            for (int s0 = cb; s0 < ce; s0 += blockDim.x) {
                __syncthreads();
                int s = s0 + threadIdx.x;
                if (s < ce) { sx[threadIdx.x] = A.xs[s]; sy[threadIdx.x] = A.ys[s]; st[threadIdx.x] = A.taus[s]; }
                __syncthreads();
                int ns = min((int)blockDim.x, ce - s0);
                if (act)
                    for (int u = 0; u < ns; u++) {
                        double dx = px - sx[u], dy = py - sy[u];
                        if (check_self && dx == 0.0 && dy == 0.0) continue;
                        acc += green_d(A.kind, A.k, dx * dx + dy * dy) * st[u];
                    }
            }
        }
        if (act) A.pots[t] = acc;
    }
}

// L2L alone, added onto the M2L result: u_down(children of a split entry) +=
// L2L_l u_down(parent).  One warp per entry.
__global__ void k_l2l_d(PassArgs A, int l) {
    extern __shared__ double svl[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int Q = A.Q, Q4 = 4 * Q;
    double *v = svl + (size_t)wib * Q;
    bool active = e < A.T.ne[l] && !(A.ent[A.T.eoff[l] + e] & 1);
    int p = active ? A.ent_node[A.T.eoff[l] + e] : 0;
    if (active)
        for (int c = lane; c < Q; c += 32) v[c] = A.udown[(size_t)p * Q + c];
    __syncwarp();
    if (!active) return;
    int64_t c0 = A.T.off[l + 1] + 4 * e;
    const double *op = A.ops + (size_t)l * A.stride + A.off_l2l;
    for (int r = lane; r < Q4; r += 32) {
        double acc = 0.0;
        for (int c = 0; c < Q; c++) acc = fma(op[(size_t)c * Q4 + r], v[c], acc);
        A.udown[(size_t)c0 * Q + r] += acc;
    }
}

// Evaluation at arbitrary targets: locate by strict '>' descent
// (numba_locate_points, tree.py:712-727), then L2P and P2P.
__global__ void k_eval_targets_d(PassArgs A, const double *__restrict__ tx, const double *__restrict__ ty, int64_t n,
                                 int check_self, double *__restrict__ pot) {
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
        double acc = 0.0;
        if (l >= 2) {
            const double *blk = A.ops + (size_t)l * A.stride;
            const double *inv = blk + A.off_inv, *lg = blk + A.off_large;
            double rx = px - cx, ry = py - cy;
            for (int q = 0; q < A.Q; q++) {
                double qd = 0.0;
                for (int c = 0; c < A.Q; c++) qd = fma(inv[q * A.Q + c], A.udown[(size_t)g * A.Q + c], qd);
                double dx = rx - lg[q], dy = ry - lg[A.Q + q];
                acc += green_d(A.kind, A.k, dx * dx + dy * dy) * qd;
            }
        }
        for (int d = 0; d < 9; d++) {
            int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            for (int s = A.nbot[c]; s < A.ntop[c]; s++) {
                double dx = px - A.xs[s], dy = py - A.ys[s];
                if (check_self && dx == 0.0 && dy == 0.0) continue;
                acc += green_d(A.kind, A.k, dx * dx + dy * dy) * A.taus[s];
            }
        }
        pot[i] = acc;
    }
}

PassArgs make_pass_args(kifmm_plan *P) {
    PassArgs A{};
    A.T = P->lt;
    A.Q = P->Q;
    A.kind = P->kern.kind;
    A.k = P->kern.k;
    A.root = P->root_min;
    A.W = P->W;
    A.ops = P->ops.p;
    A.ops_f = P->ops_f.p;
    A.stride = P->ops_stride;
    A.off_inv = 0;
    A.off_m2m = (size_t)P->Q * P->Q;
    A.off_l2l = (size_t)5 * P->Q * P->Q;
    A.off_m2l = (size_t)9 * P->Q * P->Q;
    A.off_large = (size_t)153 * P->Q * P->Q;
    A.ent = P->ent.p;
    A.ent_node = P->ent_node.p;
    A.nkey = P->nkey.p;
    A.nlev = P->nlev.p;
    A.nflag = P->nflag.p;
    A.nbot = P->nbot.p;
    A.ntop = P->ntop.p;
    A.nchild = P->nchild.p;
    A.nent = P->nent.p;
    A.ncoll = P->ncoll.p;
    A.xs = P->xs.p;
    A.ys = P->ys.p;
    A.taus = P->taus.p;
    A.pots = P->pots.p;
    A.uup = P->uup.p;
    A.udown = P->udown.p;
    return A;
}

void launch_p2m_d(kifmm_plan *P, const PassArgs &A) {
    k_p2m_d<<<grid_for(P->n_p2m_list * 32, 256), 256, 0, P->stream>>>(A, P->p2m_list.p, P->n_p2m_list);
    KIFMM_LAUNCHED();
}

void launch_leaf_eval_d(kifmm_plan *P, const PassArgs &A, int check_self) {
    int thr = P->ppl <= 64 ? 64 : 128;
    size_t smem = (size_t)(P->Q + 3 * thr) * sizeof(double);
    k_leaf_eval_d<<<(unsigned)P->n_leaf_list, thr, smem, P->stream>>>(A, P->leaf_list.p, check_self);
    KIFMM_LAUNCHED();
}

void launch_eval_targets_d(kifmm_plan *P, const PassArgs &A, const double *tx, const double *ty, int64_t n,
                           int check_self, double *pot) {
    k_eval_targets_d<<<grid_for(n, 128, P->num_sms * 16), 128, 0, P->stream>>>(A, tx, ty, n, check_self, pot);
    KIFMM_LAUNCHED();
}

void launch_m2m_d(kifmm_plan *P, const PassArgs &A, int l) {
    int64_t ne = P->lt.ne[l];
    size_t smem = (size_t)8 * 4 * P->Q * sizeof(double);
    k_m2m_d<<<grid_for(ne * 32, 256), 256, smem, P->stream>>>(A, l);
    KIFMM_LAUNCHED();
}

void launch_l2l_d(kifmm_plan *P, const PassArgs &A, int l) {
    int64_t ne = P->lt.ne[l];
    k_l2l_d<<<grid_for(ne * 32, 256), 256, (size_t)8 * P->Q * sizeof(double), P->stream>>>(A, l);
    KIFMM_LAUNCHED();
}

void run_upward_downward(kifmm_plan *P) {
    cudaStream_t s = P->stream;
    const int Q = P->Q, L = P->L;
    int64_t n = P->N, NN = P->n_nodes;
    P->taus.alloc(n);
    P->pots.alloc(n);
    P->uup.alloc((size_t)NN * Q);
    P->udown.alloc((size_t)NN * Q);
    k_gather_tau<<<grid_for(n, 256, P->num_sms * 8), 256, 0, s>>>(P->tau.p, P->perm.p, n, P->taus.p);
    KIFMM_LAUNCHED();
    if (P->opt.precision == KIFMM_PREC_MIXED) {
        run_passes_mixed(P);
        return;
    }
    KIFMM_CUDA(cudaMemsetAsync(P->uup.p, 0, (size_t)NN * Q * sizeof(double), s));
    KIFMM_CUDA(cudaMemsetAsync(P->udown.p, 0, (size_t)NN * Q * sizeof(double), s));
    if (L < 3) return;  // no level has well-separated boxes
    PassArgs A = make_pass_args(P);
    if (P->n_p2m_list) {
        PhaseScope ph(P, KIFMM_PHASE_P2M);
        launch_p2m_d(P, A);
    }
    {
    PhaseScope ph_m2m(P, KIFMM_PHASE_M2M);
    for (int l = L - 2; l >= 2; l--) {
        int64_t ne = P->lt.ne[l];
        if (!ne) continue;
        size_t smem = (size_t)8 * 4 * Q * sizeof(double);
        k_m2m_d<<<grid_for(ne * 32, 256), 256, smem, s>>>(A, l);
        KIFMM_LAUNCHED();
    }
    }
    PhaseScope ph(P, KIFMM_PHASE_M2L);
    int thr = ((4 * Q + 31) / 32) * 32;
    size_t smem = (size_t)M2L_TE * 4 * Q * sizeof(double);
    KIFMM_CUDA(cudaFuncSetAttribute(k_m2l_d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int l = 1; l <= L - 2; l++) {
        int64_t ne = P->lt.ne[l];
        if (!ne) continue;
        k_m2l_d<<<(unsigned)((ne + M2L_TE - 1) / M2L_TE), thr, smem, s>>>(A, l);
        KIFMM_LAUNCHED();
    }
}

void run_eval_sources(kifmm_plan *P, int check_self) {
    cudaStream_t s = P->stream;
    int64_t n = P->N;
    P->pot_out.alloc(n);
    if (P->opt.precision == KIFMM_PREC_MIXED) {
        run_eval_sources_mixed(P, check_self);
    } else {
        PassArgs A = make_pass_args(P);
        if (P->n_leaf_list) {
            PhaseScope ph(P, KIFMM_PHASE_LEAF);
            launch_leaf_eval_d(P, A, check_self);
        }
    }
    k_scatter_pot<<<grid_for(n, 256, P->num_sms * 8), 256, 0, s>>>(P->pots.p, P->perm.p, n, P->pot_out.p);
    KIFMM_LAUNCHED();
}

void run_eval_targets(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self, double *pot) {
    PassArgs A = make_pass_args(P);
    if (P->opt.precision == KIFMM_PREC_MIXED) {
        run_eval_targets_mixed(P, tx, ty, n, check_self, pot);
        return;
    }
    launch_eval_targets_d(P, A, tx, ty, n, check_self, pot);
}

// ------------------------------------------------ kernel-function utilities
// KAS restricted to targets (class_fmm.py:134-143): one block per target.
__global__ void k_direct_d(int kind, double k, const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ tau, int64_t n, const int64_t *__restrict__ tg,
                           double *__restrict__ out) {
    __shared__ double red[32];
    int64_t j = tg[blockIdx.x];
    if (j < 0 || j >= n) {  // caller index out of range: report NaN, touch nothing
        if (threadIdx.x == 0) out[blockIdx.x] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    double px = x[j], py = y[j], acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        if (i == j) continue;
        double dx = px - x[i], dy = py - y[i];
        acc += green_d(kind, k, dx * dx + dy * dy) * tau[i];
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) out[blockIdx.x] = v;
    }
}

__global__ void k_kmatrix_d(int kind, double k, const double *sx, const double *sy, int64_t ns, const double *tx,
                            const double *ty, int64_t nt, double *out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ns * nt; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = e / ns, i = e % ns;
        double dx = tx[j] - sx[i], dy = ty[j] - sy[i];
        out[e] = green_d(kind, k, dx * dx + dy * dy);
    }
}

__global__ void k_kapply_d(int kind, double k, const double *sx, const double *sy, int64_t ns, const double *tx,
                           const double *ty, int64_t nt, const double *tau, double *out) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nt; j += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int64_t i = 0; i < ns; i++) {
            double dx = tx[j] - sx[i], dy = ty[j] - sy[i];
            acc += green_d(kind, k, dx * dx + dy * dy) * tau[i];
        }
        out[j] = acc;
    }
}

void direct_sum_device(const kifmm_kernel &kn, const double *x, const double *y, const double *tau, int64_t n,
                       const int64_t *tg, int64_t nt, double *out, cudaStream_t s) {
    if (nt <= 0) return;
    KIFMM_REQUIRE(nt < (1ll << 31), KIFMM_ERR_ARG, "direct_sum: too many targets");
    k_direct_d<<<(unsigned)nt, 256, 0, s>>>(kn.kind, kn.k, x, y, tau, n, tg, out);
    KIFMM_LAUNCHED();
}

void kernel_matrix_device(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                          const double *ty, int64_t nt, double *out, cudaStream_t s) {
    if (ns * nt <= 0) return;
    k_kmatrix_d<<<grid_for(ns * nt, 256, 8192), 256, 0, s>>>(kn.kind, kn.k, sx, sy, ns, tx, ty, nt, out);
    KIFMM_LAUNCHED();
}

void kernel_apply_device(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                         const double *ty, int64_t nt, const double *tau, double *out, cudaStream_t s) {
    if (nt <= 0) return;
    k_kapply_d<<<grid_for(nt, 128, 8192), 128, 0, s>>>(kn.kind, kn.k, sx, sy, ns, tx, ty, nt, tau, out);
    KIFMM_LAUNCHED();
}

}  // namespace kifmm
