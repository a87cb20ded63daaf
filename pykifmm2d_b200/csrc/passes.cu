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
#include "async_copy.cuh"

namespace kifmm {

__global__ void k_gather_tau(const double *__restrict__ tau, const int32_t *__restrict__ perm, int64_t n,
                             double *__restrict__ taus) {
    pdl_trigger();
    pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        taus[i] = tau[perm[i]];
}

__global__ void k_scatter_pot(const double *__restrict__ pots, const int32_t *__restrict__ perm, int64_t n,
                              double *__restrict__ pot) {
    pdl_trigger();
    pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pot[perm[i]] = pots[i];
}

// Natural logarithm for the Laplace P2M sums, table-driven (P. T. P. Tang,
// "Table-driven implementation of the logarithm function in IEEE
// floating-point arithmetic", ACM TOMS 16, 1990): x = 2^e m with m in [1, 2),
// c_i = 1 + (i + 1/2)/128 the midpoint of m's subinterval, r = m / c_i - 1
// (|r| < 2^-8), ln x = e ln2 + ln c_i + log1p(r) with log1p by its series to
// r^7 (the next term is below 2^-67).  ln c_i and 1/c_i are computed on the
// host in long double (init_log_table) and staged in shared memory.
__device__ double g_logtab[256];  // [0..127] ln c_i, [128..255] 1 / c_i
constexpr double LN2_HI = 6.93147180369123816490e-01, LN2_LO = 1.90821492927058770002e-10;
__device__ __forceinline__ double ln_tab(double x, const double *lt) {
    const long long b = __double_as_longlong(x);
    const int e = (int)((b >> 52) & 0x7ff) - 1023;
    const int i = (int)((b >> 45) & 127);
    const double m = __longlong_as_double((b & 0x000fffffffffffffll) | 0x3ff0000000000000ll);
    const double r = fma(m, lt[128 + i], -1.0);
    double p = 1.0 / 7.0;
    p = fma(p, r, -1.0 / 6.0);
    p = fma(p, r, 1.0 / 5.0);
    p = fma(p, r, -1.0 / 4.0);
    p = fma(p, r, 1.0 / 3.0);
    p = fma(p, r, -0.5);
    p = fma(p * r, r, r);  // r + r^2 (-1/2 + r (1/3 - ...))
    return fma((double)e, LN2_HI, lt[i] + fma((double)e, LN2_LO, p));
}
void init_log_table(int device) {
    static bool done[64] = {};
    if (device < 0 || device >= 64 || done[device]) return;
    double t[256];
    for (int i = 0; i < 128; i++) {
        const long double c = 1.0L + ((long double)i + 0.5L) / 128.0L;
        t[i] = (double)logl(c);
        t[128 + i] = (double)(1.0L / c);
    }
    KIFMM_CUDA(cudaMemcpyToSymbol(g_logtab, t, sizeof(t)));
    done[device] = true;
}

// P2M (numba_upwards_pass, class_fmm.py:57-71): one warp per node; lane q
// accumulates over the node's sources, which the warp stages 32 at a time
// in shared memory.  Laplace sums tau log(r^2) with ln_tab and scales once.
constexpr int P2M_WARPS = 8;
__global__ void __launch_bounds__(32 * P2M_WARPS) k_p2m_d(PassArgs A, const int32_t *__restrict__ list,
                                                           int64_t nlist) {
    __shared__ double sx[P2M_WARPS][32], sy[P2M_WARPS][32], st[P2M_WARPS][32];
    __shared__ double lt[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lt[i] = g_logtab[i];
    __syncthreads();
    pdl_trigger();
    pdl_wait();
    const bool lap = A.kind == KIFMM_KERNEL_LAPLACE;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= nlist) return;
    int g = list[w];
    int l = A.nlev[g];
    double cx, cy;
    node_center(A, g, l, cx, cy);
    const double *lg = A.ops + (size_t)l * A.stride + A.off_large;
    const int b = A.nbot[g], e = A.ntop[g];
    for (int q0 = 0; q0 < A.Q; q0 += 32) {
        int q = q0 + lane;
        bool ok = q < A.Q;
        double tx = ok ? lg[q] + cx : 0.0, ty = ok ? lg[A.Q + q] + cy : 0.0;
        double acc0 = 0.0, acc1 = 0.0;
        for (int s0 = b; s0 < e; s0 += 32) {
            __syncwarp();
            if (s0 + lane < e) {
                sx[wib][lane] = A.xs[s0 + lane];
                sy[wib][lane] = A.ys[s0 + lane];
                st[wib][lane] = A.taus[s0 + lane];
            }
            __syncwarp();
            const int ns = min(32, e - s0);
            int u = 0;
            if (lap) {
                for (; u + 1 < ns; u += 2) {
                    double dx0 = tx - sx[wib][u], dy0 = ty - sy[wib][u];
                    double dx1 = tx - sx[wib][u + 1], dy1 = ty - sy[wib][u + 1];
                    acc0 = fma(ln_tab(dx0 * dx0 + dy0 * dy0, lt), st[wib][u], acc0);
                    acc1 = fma(ln_tab(dx1 * dx1 + dy1 * dy1, lt), st[wib][u + 1], acc1);
                }
                if (u < ns) {
                    double dx = tx - sx[wib][u], dy = ty - sy[wib][u];
                    acc0 = fma(ln_tab(dx * dx + dy * dy, lt), st[wib][u], acc0);
                }
            } else {
                for (; u + 1 < ns; u += 2) {
                    double dx0 = tx - sx[wib][u], dy0 = ty - sy[wib][u];
                    double dx1 = tx - sx[wib][u + 1], dy1 = ty - sy[wib][u + 1];
                    acc0 += green_d(A.kind, A.k, dx0 * dx0 + dy0 * dy0) * st[wib][u];
                    acc1 += green_d(A.kind, A.k, dx1 * dx1 + dy1 * dy1) * st[wib][u + 1];
                }
                if (u < ns) {
                    double dx = tx - sx[wib][u], dy = ty - sy[wib][u];
                    acc0 += green_d(A.kind, A.k, dx * dx + dy * dy) * st[wib][u];
                }
            }
        }
        // Laplace: G = -log(r^2) / (4 pi)
        if (ok) A.uup[(size_t)g * A.Q + q] = lap ? -0.07957747154594767 * (acc0 + acc1) : acc0 + acc1;
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
                const int je = m2l_source_entry(A.ncoll, A.nent, A.nbot, A.ntop, p, d);
                if (je >= 0) grp = A.T.off[l + 1] + 4 * (je - A.T.eoff[l]);
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

// M2L of every level in one launch on the FP64 tensor path (mma.sync
// m8n8k4 .f64), class_fmm.py:336-343 recast target-centric:
//   u_down(children of p) = sum_{d != centre} C_d . u_up(children of p + d),
// C_d = CM2LS_d . blockdiag(Inv) (4Q x 4Q, column-major).  A block owns 32
// consecutive split entries of one level (its target groups) and all 4Q rows:
// D[4Q x 32] = sum over (direction, K chunk of 32) of C_d[:, chunk] .
// B_d[chunk, 32], B_d's columns the targets' source groups in direction d
// (a zero vector where a target has none).  Stages run through a ring of two
// shared-memory slots, warp-specialised: a copy warp fills a slot by bulk
// copies (the operator chunk as 32 columns of 4Q doubles, the sources as 32
// rows of 32 doubles, one copy per lane) on the slot's full barrier as soon
// as the eight compute warps have arrived on its empty barrier, so the
// copies of stage s + 1 land while stage s computes and no block-wide
// barrier stands in the loop.  Compute warp w owns row tiles w, w + 8, ...
// (8 rows each) for all 32 targets.  D is assigned to the
// children's u_down (the L2L chain adds afterwards).  Needs Q even.
#ifndef KIFMM_MD_KC
#define KIFMM_MD_KC 32
#endif
#ifndef KIFMM_MD_NBUF
#define KIFMM_MD_NBUF 2
#endif
constexpr int MD_THREADS = 256, MD_TE = 32, MD_KC = KIFMM_MD_KC, MD_MT = 4;  // Q4 <= 8 warps x MD_MT x 8 rows
constexpr int MD_NBUF = KIFMM_MD_NBUF;  // ring slots: copies run MD_NBUF - 1 stages ahead
constexpr int MD_BLOCK = MD_THREADS + 32;  // eight compute warps and one copy warp
static_assert(MD_KC % 4 == 0 && MD_NBUF >= 2 && MD_NBUF <= 8, "DMMA M2L staging shape");
struct M2lDmmaArgs {
    PassArgs A;
    const double *zero;                 // 4Q zeros
    int lmin, lmax;
    int64_t tile_off[MAX_LEVELS + 1];   // first block of each parent level
    long long wait_limit;
    unsigned long long *err;
};
// warp-uniform bounded wait on an mbarrier phase (every lane polls; true
// once the phase has completed, false after `limit` polls)
__device__ __forceinline__ bool warp_wait_all(uint32_t bar, uint32_t parity, long long limit) {
    return __any_sync(0xffffffffu, mbar_wait(bar, parity, limit));
}
static size_t m2l_dmma_smem(int Q4) {
    const size_t ldo = pad4mod16(Q4), ldx = pad4mod16(MD_KC);
    const size_t stage = (size_t)MD_KC * ldo + (size_t)MD_TE * ldx;
    const size_t out = (size_t)MD_TE * (Q4 + 1);
    return (MD_NBUF * stage > out ? MD_NBUF * stage : out) * sizeof(double) + MD_TE * 8 * sizeof(int) + 64;
}
__global__ void __launch_bounds__(MD_BLOCK, 2) k_m2l_dmma(M2lDmmaArgs M) {
    extern __shared__ __align__(128) double sm_md[];
    const PassArgs &A = M.A;
    const int Q = A.Q, Q4 = 4 * Q, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ldo = pad4mod16(Q4), ldx = pad4mod16(MD_KC);
    const size_t stage_d = (size_t)MD_KC * ldo + (size_t)MD_TE * ldx;
    int *ssrc = (int *)(sm_md + (MD_NBUF * stage_d > (size_t)MD_TE * (Q4 + 1) ? MD_NBUF * stage_d
                                                                              : (size_t)MD_TE * (Q4 + 1)));
    __shared__ __align__(8) uint64_t bars[MD_NBUF], empty[MD_NBUF];
    __shared__ int sabort;
    __shared__ int sact[MD_TE];
    __shared__ int sdir[8], scm[8], snd;  // active directions, their 8-target column tiles with a source
    pdl_trigger();
    const int64_t b = blockIdx.x;
    int l = M.lmin;
    while (l < M.lmax && M.tile_off[l + 1] <= b) l++;
    const int64_t e0 = (b - M.tile_off[l]) * MD_TE, ne = A.T.ne[l], eoff = A.T.eoff[l];
    const double *opl = A.ops + (size_t)(l + 1) * A.stride + A.off_m2l;  // target level's operators
    pdl_wait();  // u_up comes from the M2M chain
    if (tid < MD_TE) {  // the tile's targets in M2L target order; sact = 1 + index in the level, 0: none
        const int64_t e = e0 + tid, ej = e < ne ? (int64_t)A.m2l_perm[eoff + e] : -1;
        const bool act = ej >= 0 && !(A.ent[ej] & 1);
        sact[tid] = act ? (int)(ej - eoff) + 1 : 0;
        for (int dd = 0; dd < 8; dd++) ssrc[tid * 8 + dd] = act ? A.m2l_src8[ej * 8 + dd] : -1;
    }
    if (tid == 0) {
        for (int i = 0; i < MD_NBUF; i++) {
            mbar_init(smem_u32(&bars[i]));              // full: the stage's copies (transaction bytes)
            mbar_init(smem_u32(&empty[i]), MD_THREADS / 32);  // empty: each compute warp is done with it
        }
        sabort = 0;
    }
    __syncthreads();
    // Work skipped: a direction no target of the block has a source in, and
    // within a direction each 8-target column tile without one (a V-list
    // group is absent where the colleague is missing, a leaf or empty).
    if (tid < 8) {
        int m = 0;
        for (int n = 0; n < MD_TE; n++) m |= (ssrc[n * 8 + tid] >= 0) << (n >> 3);
        scm[tid] = m;
    }
    __syncthreads();
    if (tid == 0) {
        int k = 0;
        for (int dd = 0; dd < 8; dd++)
            if (scm[dd]) sdir[k++] = dd;
        snd = k;
    }
    __syncthreads();
    const int nkc = (Q4 + MD_KC - 1) / MD_KC, nst = snd * nkc;
    // the lanes of warp 0 issue the copies of stage st into buffer st % 2
    // (one operator column and one source row each: issued by one thread
    // they kept warp 0, and the whole block at the next barrier, waiting)
    auto issue = [&](int st) {
        const int dd = sdir[st / nkc], d = dd < 4 ? dd : dd + 1, kc = st % nkc, k0 = kc * MD_KC;
        const int kn = min(MD_KC, Q4 - k0), cm = scm[dd];
        double *bs = sm_md + (size_t)(st % MD_NBUF) * stage_d;
        const uint32_t bar = smem_u32(&bars[st % MD_NBUF]);
        if (lane == 0) mbar_expect_tx(bar, (uint32_t)(kn * Q4 + 8 * __popc(cm) * kn) * 8u);
        __syncwarp();
        const double *op = opl + (size_t)d * Q4 * Q4 + (size_t)k0 * Q4;
        for (int c = lane; c < kn; c += 32)
            bulk_g2s(smem_u32(bs + (size_t)c * ldo), op + (size_t)c * Q4, (uint32_t)Q4 * 8u, bar);
        double *xs = bs + (size_t)MD_KC * ldo;
        for (int n = lane; n < MD_TE; n += 32) {
            if (!((cm >> (n >> 3)) & 1)) continue;
            const int je = ssrc[n * 8 + dd];
            const double *src = je >= 0 ? A.uup + (size_t)(A.T.off[l + 1] + 4 * (je - eoff)) * Q + k0 : M.zero + k0;
            bulk_g2s(smem_u32(xs + (size_t)n * ldx), src, (uint32_t)kn * 8u, bar);
        }
    };
    const int g = lane >> 2, t = lane & 3, nrt = Q4 / 8;
    double acc[MD_MT][4][2];
#pragma unroll
    for (int i = 0; i < MD_MT; i++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[i][c][0] = acc[i][c][1] = 0.0;
    volatile int *abort_flag = &sabort;
    if (warp == MD_THREADS / 32) {
        // producer warp: stage st goes into slot st % MD_NBUF once the compute
        // warps have released the slot's previous stage
        int issued = 0;
        for (int st = 0; st < nst; st++) {
            const int slot = st % MD_NBUF;
            if (st >= MD_NBUF && !warp_wait_all(smem_u32(&empty[slot]), (uint32_t)(st / MD_NBUF - 1) & 1u, M.wait_limit)) {
                if (lane == 0) {
                    *abort_flag = 1;
                    atomicOr(M.err, 1ull);
                }
                break;
            }
            if (*abort_flag) break;
            issue(st);
            issued = st + 1;
        }
        // every copy issued lands before the block goes on (consumed stages
        // have landed already; this matters after an abort)
        for (int st = issued > MD_NBUF ? issued - MD_NBUF : 0; st < issued; st++)
            mbar_wait(smem_u32(&bars[st % MD_NBUF]), (uint32_t)(st / MD_NBUF) & 1u, kDrainWaitPolls);
    } else {
        for (int st = 0; st < nst; st++) {
            const int bi = st % MD_NBUF;
            if (!warp_wait_all(smem_u32(&bars[bi]), (uint32_t)(st / MD_NBUF) & 1u, M.wait_limit)) {
                if (lane == 0) {
                    *abort_flag = 1;
                    atomicOr(M.err, 1ull);
                }
                break;
            }
            if (*abort_flag) break;
            const int kn = min(MD_KC, Q4 - (st % nkc) * MD_KC), cm = scm[sdir[st / nkc]];
            const double *os = sm_md + (size_t)bi * stage_d, *xs = os + (size_t)MD_KC * ldo;
            for (int k0 = 0; k0 < kn; k0 += 4) {
                double bv[4];
#pragma unroll
                for (int c = 0; c < 4; c++) bv[c] = xs[(size_t)(8 * c + g) * ldx + k0 + t];
#pragma unroll
                for (int i = 0; i < MD_MT; i++) {
                    const int rt = warp + 8 * i;
                    if (rt < nrt) {
                        const double av = os[(size_t)(k0 + t) * ldo + 8 * rt + g];
#pragma unroll
                        for (int c = 0; c < 4; c++)
                            if ((cm >> c) & 1) dmma_8x8x4(acc[i][c][0], acc[i][c][1], av, bv[c]);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&empty[bi]));  // this warp is done with the slot
        }
    }
    __syncthreads();
    if (*abort_flag) return;
    // D through shared memory (the stage buffers are free), then coalesced stores
    double *cs = sm_md;  // [32 targets][Q4 + 1]
#pragma unroll
    for (int i = 0; i < MD_MT; i++) {
        const int rt = warp + 8 * i;
        if (warp < MD_THREADS / 32 && rt < nrt)
#pragma unroll
            for (int c = 0; c < 4; c++) {
                cs[(size_t)(8 * c + 2 * t) * (Q4 + 1) + 8 * rt + g] = acc[i][c][0];
                cs[(size_t)(8 * c + 2 * t + 1) * (Q4 + 1) + 8 * rt + g] = acc[i][c][1];
            }
    }
    __syncthreads();
    for (int n = warp; n < MD_TE; n += MD_BLOCK / 32) {
        if (!sact[n]) continue;
        double *dst = A.udown + ((size_t)A.T.off[l + 1] + 4 * (size_t)(sact[n] - 1)) * Q;
        for (int r = lane; r < Q4; r += 32) dst[r] = cs[(size_t)n * (Q4 + 1) + r];
    }
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

// Evaluation at arbitrary targets: locate by strict '>' descent
// (numba_locate_points, tree.py:712-727), then L2P and P2P.
// Targets in Morton order (sort_targets) with the leaves' equivalent densities
// precomputed (k_leaf_den); out[order[i]] is target i's potential.
__global__ void k_eval_targets_d(PassArgs A, const double *__restrict__ tx, const double *__restrict__ ty, int64_t n,
                                 int check_self, const int32_t *__restrict__ order, const double *__restrict__ den,
                                 double *__restrict__ pot) {
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
            const double *lg = blk + A.off_large;
            double rx = px - cx, ry = py - cy;
            const double *dg = den + (size_t)g * A.Q;
            for (int q = 0; q < A.Q; q++) {
                double dx = rx - lg[q], dy = ry - lg[A.Q + q];
                acc += green_d(A.kind, A.k, dx * dx + dy * dy) * dg[q];
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
        pot[order[i]] = acc;
    }
}

PassArgs make_pass_args(kifmm_plan *P) {
    PassArgs A{};
    A.T = P->lt;
    A.Q = P->Q;
    A.Qc = P->Qc;
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
    A.leaf_rec = P->leaf_rec.p;
    A.m2l_perm = P->m2l_perm.p;
    A.m2l_src8 = P->m2l_src8.p;
    A.taylor = P->l2p_taylor.p;
    A.leaf_coef = P->leaf_coef.p;
    return A;
}

__global__ void k_leaf_records(PassArgs A, const int32_t *__restrict__ leaves, int64_t n, int32_t *__restrict__ rec) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int g = leaves[i];
        int r[LEAF_REC_WORDS] = {};
        r[LR_NODE] = g;
        r[LR_LEVEL] = A.nlev[g];
        r[LR_BOT] = A.nbot[g];
        r[LR_TOP] = A.ntop[g];
        const uint64_t k = A.nkey[g];
        r[LR_KEY_LO] = (int32_t)(uint32_t)k;
        r[LR_KEY_HI] = (int32_t)(uint32_t)(k >> 32);
        r[LR_NSRC] = leaf_ranges(A, g, r + LR_RNG);
        int4 *o = (int4 *)(rec + i * LEAF_REC_WORDS);
#pragma unroll
        for (int q = 0; q < LEAF_REC_WORDS / 4; q++) o[q] = make_int4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
    }
}

// the leaf records of the plan's leaf list (part of the tree build)
void build_leaf_records(kifmm_plan *P) {
    P->leaf_rec.alloc((size_t)(P->n_leaf_list ? P->n_leaf_list : 1) * LEAF_REC_WORDS);
    if (!P->n_leaf_list) return;
    PassArgs A = make_pass_args(P);
    k_leaf_records<<<grid_for(P->n_leaf_list, 128, P->num_sms * 8), 128, 0, P->stream>>>(
        A, P->leaf_list.p, P->n_leaf_list, P->leaf_rec.p);
    KIFMM_LAUNCHED();
}

// M2L target order.  The entries of each level are grouped by the set of
// directions in which they have V-list sources (an 8-bit mask; entries that
// are not split go last), so that an M2L tile of consecutive targets mostly
// shares one set and skips every absent direction instead of multiplying
// zero vectors.  The mask depends on the tree only: the order is built once
// per tree.  Within a group the order is whatever the atomics give; the M2L
// result of a target does not depend on which other targets share its tile.
__global__ void k_m2l_keys(PassArgs A, int64_t n_ent, uint16_t *__restrict__ key, int32_t *__restrict__ src8,
                           unsigned *__restrict__ hist) {
    pdl_trigger();
    pdl_wait();
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool in = j < n_ent;
    unsigned bin = 0xffffffffu;
    if (in) {
        const uint64_t ej = A.ent[j];
        const int l = (int)(ej >> ENT_LEVEL_SHIFT);
        const bool split = !(ej & 1);
        int k = split ? 0 : 256, sv[8];
#pragma unroll
        for (int dd = 0; dd < 8; dd++) {
            const int d = dd < 4 ? dd : dd + 1;
            sv[dd] = split ? m2l_source_entry(A.ncoll, A.nent, A.nbot, A.ntop, A.ent_node[j], d) : -1;
            if (sv[dd] >= 0) k |= 1 << dd;
        }
        int4 *o = (int4 *)(src8 + 8 * j);
        o[0] = make_int4(sv[0], sv[1], sv[2], sv[3]);
        o[1] = make_int4(sv[4], sv[5], sv[6], sv[7]);
        key[j] = (uint16_t)k;
        bin = (unsigned)(l * M2L_KEYS + k);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (in && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[bin], (unsigned)__popc(peers));
}

// counts -> first position of each (level, key) group, from the level's
// eoff: one block per level, an exclusive scan over the 257 keys
constexpr int M2L_SCAN_THREADS = 288;  // >= M2L_KEYS, a whole number of warps
__global__ void __launch_bounds__(M2L_SCAN_THREADS) k_m2l_cursors(LevelTable T, unsigned *__restrict__ hist) {
    __shared__ unsigned wsum[M2L_SCAN_THREADS / 32];
    pdl_trigger();
    pdl_wait();
    const int l = blockIdx.x, k = threadIdx.x, lane = k & 31, w = k >> 5;
    const unsigned c = k < M2L_KEYS ? hist[l * M2L_KEYS + k] : 0u;
    unsigned v = c;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) wsum[w] = v;
    __syncthreads();
    unsigned before = (unsigned)T.eoff[l];
    for (int i = 0; i < w; i++) before += wsum[i];
    if (k < M2L_KEYS) hist[l * M2L_KEYS + k] = before + v - c;
}

__global__ void k_m2l_place(const uint64_t *__restrict__ ent, const uint16_t *__restrict__ key, int64_t n_ent,
                            unsigned *__restrict__ cursor, int32_t *__restrict__ perm) {
    pdl_trigger();
    pdl_wait();
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool in = j < n_ent;
    const int lane = threadIdx.x & 31;
    const unsigned bin = in ? (unsigned)((int)(ent[j] >> ENT_LEVEL_SHIFT) * M2L_KEYS + key[j]) : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    const int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (in && lane == leader) base = atomicAdd(&cursor[bin], (unsigned)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (in) perm[base + __popc(peers & ((1u << lane) - 1))] = (int32_t)j;
}

void build_m2l_order(kifmm_plan *P) {
    const int64_t n = P->n_ent;
    P->m2l_perm.alloc(n ? n : 1);
    if (!n) return;
    KIFMM_REQUIRE(P->L <= MAX_LEVELS + 1 && n < (1ll << 31), KIFMM_ERR_ARG, "M2L order: tree too large");
    P->m2l_key.alloc(n);
    P->m2l_src8.alloc((size_t)8 * n);
    // m2l_hist ([MAX_LEVELS + 1][M2L_KEYS] counts) is allocated and cleared by
    // build_tree with the split-cell set
    PassArgs A = make_pass_args(P);
    const unsigned gr = (unsigned)((n + 255) / 256);
    launch_pdl(k_m2l_keys, dim3(gr), dim3(256), 0, P->stream, A, n, P->m2l_key.p, P->m2l_src8.p, P->m2l_hist.p);
    launch_pdl(k_m2l_cursors, dim3((unsigned)std::min(P->L, MAX_LEVELS + 1)), dim3(M2L_SCAN_THREADS), 0, P->stream,
               P->lt, P->m2l_hist.p);
    launch_pdl(k_m2l_place, dim3(gr), dim3(256), 0, P->stream, (const uint64_t *)P->ent.p,
               (const uint16_t *)P->m2l_key.p, n, P->m2l_hist.p, P->m2l_perm.p);
    KIFMM_LAUNCHED();
}

void launch_p2m_d(kifmm_plan *P, const PassArgs &A) {
launch_pdl(k_p2m_d, dim3(grid_for(P->n_p2m_list * 32, 32 * P2M_WARPS)), dim3(32 * P2M_WARPS), 0, P->stream, A,
               (const int32_t *)P->p2m_list.p, P->n_p2m_list);
}

void launch_leaf_eval_d(kifmm_plan *P, const PassArgs &A, int check_self) {
    int thr = P->ppl <= 64 ? 64 : 128;
    size_t smem = (size_t)(P->Q + 3 * thr) * sizeof(double);
    k_leaf_eval_d<<<(unsigned)P->n_leaf_list, thr, smem, P->stream>>>(A, P->leaf_list.p, check_self);
    KIFMM_LAUNCHED();
}

void sort_targets(kifmm_plan *P, const double *tx, const double *ty, int64_t n);  // tree.cu
void launch_leaf_den(kifmm_plan *P, const PassArgs &A);                          // passes_mixed.cu

void launch_eval_targets_d(kifmm_plan *P, const PassArgs &A, const double *tx, const double *ty, int64_t n,
                           int check_self, double *pot) {
    sort_targets(P, tx, ty, n);
    launch_leaf_den(P, A);
    k_eval_targets_d<<<grid_for(n, 128, P->num_sms * 16), 128, 0, P->stream>>>(
        A, P->txs.p, P->tys.p, n, check_self, P->tperm.p, P->node_den.p, pot);
    KIFMM_LAUNCHED();
}

// M2M and L2L as small FP64 GEMMs per level, C[M x n] = Op[M x K] X[K x n]:
//   M2M: M = Q, K = 4Q, X = the entries' children groups (contiguous), C -> the
//        entries' own rows of u_up;
//   L2L: M = 4Q, K = Q, X = the split entries' u_down (gathered), C added to
//        their children groups.
// A block stages the whole operator and NT columns of X in shared memory and
// each thread accumulates a 4 x 4 register tile.
template <int MODE>
__global__ void __launch_bounds__(256) k_lvl_gemm_d(PassArgs A, int l, int M, int K, int NT) {
    extern __shared__ double sm_g[];
    double *opS = sm_g;                       // [K][M]
    double *xS = sm_g + (size_t)K * M;        // [NT][K + 1]
    const int ldx = K + 1;
    const int Q = A.Q;
    const int64_t ne = A.T.ne[l], eoff = A.T.eoff[l], e0 = (int64_t)blockIdx.x * NT;
    const double *op = A.ops + (size_t)l * A.stride + (MODE == 0 ? A.off_m2m : A.off_l2l);
    // operator: 16-byte loads when aligned (odd Nequiv gives odd offsets)
    if ((((uintptr_t)op) & 15) == 0 && (K * M) % 2 == 0)
        for (int i = threadIdx.x; i < K * M / 2; i += blockDim.x) ((double2 *)opS)[i] = ((const double2 *)op)[i];
    else
        for (int i = threadIdx.x; i < K * M; i += blockDim.x) opS[i] = op[i];
    const double *src0 = A.uup + (size_t)(A.T.off[l + 1] + 4 * e0) * Q;
    if (MODE == 0 && (((uintptr_t)src0) & 15) == 0) {  // children groups of consecutive entries: one block
        const int64_t nt = min((int64_t)NT, ne - e0);
        const double2 *src = (const double2 *)src0;
        for (int i = threadIdx.x; i < NT * K / 2; i += blockDim.x) {
            int t = (2 * i) / K, c = (2 * i) % K;
            double2 v = t < nt ? src[i] : make_double2(0.0, 0.0);
            xS[t * ldx + c] = v.x;
            xS[t * ldx + c + 1] = v.y;
        }
    } else {
        for (int i = threadIdx.x; i < NT * K; i += blockDim.x) {
            int t = i / K, c = i % K;
            int64_t e = e0 + t;
            double v = 0.0;
            if (e < ne) {
                if (MODE == 0) v = src0[(size_t)t * K + c];
                else if (!(A.ent[eoff + e] & 1)) v = A.udown[(size_t)A.ent_node[eoff + e] * Q + c];
            }
            xS[t * ldx + c] = v;
        }
    }
    __syncthreads();
    const int TMr = (M + 3) / 4;
    const int tx = threadIdx.x % TMr, ty = threadIdx.x / TMr;
    if (ty * 4 >= NT) return;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    const int r0 = tx * 4;
    for (int c = 0; c < K; c++) {
        double a[4], bb[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = r0 + i < M ? opS[c * M + r0 + i] : 0.0;
#pragma unroll
        for (int j = 0; j < 4; j++) bb[j] = xS[(ty * 4 + j) * ldx + c];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int64_t e = e0 + ty * 4 + j;
        if (e >= ne) continue;
        if (MODE == 0) {
            double *dst = A.uup + (size_t)A.ent_node[eoff + e] * Q;
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (r0 + i < M) dst[r0 + i] = acc[i][j];
        } else {
            if (A.ent[eoff + e] & 1) continue;
            double *dst = A.udown + (size_t)(A.T.off[l + 1] + 4 * e) * Q;
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (r0 + i < M) dst[r0 + i] += acc[i][j];
        }
    }
}

// The same products with the operator held once per block and one entry per
// lane: warp w of a block takes 32 entries and RPT rows of the operator, so
// every operator read is a shared-memory broadcast (two rows per 16-byte
// load) and each thread's RPT accumulators are FP64-pipe bound.  Rows are
// padded to Mp = RG * RPT with zeros.  Blocks hold NT = 32 * S entries, S
// sets of wps = min(RG, 8) warps; with RG > 8 a warp loops over row groups.
constexpr int LG_THREADS = 256;

// Copy n doubles from global memory through store(i, v), i in [0, n), with
// eight independent loads per thread in flight (16-byte loads when src is
// 16-byte aligned and n even).  Small staging loops are otherwise bound by
// one load latency per iteration.
template <int NTHR, class F>
__device__ __forceinline__ void stage_f64(const double *__restrict__ src, int n, F store) {
    if ((((uintptr_t)src) & 15) == 0 && (n & 1) == 0) {
        const double2 *s2 = (const double2 *)src;
        const int n2 = n >> 1;
        for (int i0 = threadIdx.x; i0 < n2; i0 += 8 * NTHR) {
            double2 v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = i0 + k * NTHR;
                v[k] = i < n2 ? s2[i] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = i0 + k * NTHR;
                if (i < n2) {
                    store(2 * i, v[k].x);
                    store(2 * i + 1, v[k].y);
                }
            }
        }
    } else {
        for (int i0 = threadIdx.x; i0 < n; i0 += 8 * NTHR) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = i0 + k * NTHR;
                v[k] = i < n ? src[i] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = i0 + k * NTHR;
                if (i < n) store(i, v[k]);
            }
        }
    }
}
template <int MODE, int RPT>
__global__ void __launch_bounds__(LG_THREADS) k_lvl_gemm_b(PassArgs A, int l, int M, int K, int Mp, int NT) {
    extern __shared__ __align__(16) double sm_b[];
    double *opS = sm_b;                    // [K][Mp]
    double *xS = sm_b + (size_t)K * Mp;    // [NT][K + 1]
    const int ldx = K + 1, Q = A.Q;
    const int64_t ne = A.T.ne[l], eoff = A.T.eoff[l], e0 = (int64_t)blockIdx.x * NT;
    const int nt = (int)min((int64_t)NT, ne - e0);
    const double *op = A.ops + (size_t)l * A.stride + (MODE == 0 ? A.off_m2m : A.off_l2l);  // [K][M]
    // staging: eight independent loads per thread in flight
    if (Mp != M)
        for (int i = threadIdx.x; i < K * Mp; i += LG_THREADS) opS[i] = 0.0;
    stage_f64<LG_THREADS>(op, K * M, [&](int i, double v) {
        const int c = i / M;
        opS[c * Mp + (i - c * M)] = v;
    });
    if (MODE == 0) {  // children groups of consecutive entries are contiguous
        const double *src0 = A.uup + (size_t)(A.T.off[l + 1] + 4 * e0) * Q;
        for (int i = nt * K + threadIdx.x; i < NT * K; i += LG_THREADS) {
            const int t = i / K;
            xS[t * ldx + (i - t * K)] = 0.0;
        }
        stage_f64<LG_THREADS>(src0, nt * K, [&](int i, double v) {
            const int t = i / K;
            xS[t * ldx + (i - t * K)] = v;
        });
    } else {
        for (int i0 = threadIdx.x; i0 < NT * K; i0 += 8 * LG_THREADS) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = i0 + k * LG_THREADS, t = i / K;
                v[k] = 0.0;
                if (i < NT * K && t < nt && !(A.ent[eoff + e0 + t] & 1))
                    v[k] = A.udown[(size_t)A.ent_node[eoff + e0 + t] * Q + (i - t * K)];
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int i = i0 + k * LG_THREADS, t = i / K;
                if (i < NT * K) xS[t * ldx + (i - t * K)] = v[k];
            }
        }
    }
    __syncthreads();
    const int RG = Mp / RPT, wps = RG < 8 ? RG : 8, S = 8 / wps;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int set = warp / wps;
    if (set >= S) return;
    const int t = set * 32 + lane;
    const double *xp = xS + (size_t)t * ldx;
    for (int rg = warp % wps; rg < RG; rg += wps) {
        double acc[RPT];
#pragma unroll
        for (int i = 0; i < RPT; i++) acc[i] = 0.0;
        const double *ap = opS + rg * RPT;
#pragma unroll 2
        for (int c = 0; c < K; c++) {
            const double xv = xp[c];
            const double2 *a2 = (const double2 *)(ap + (size_t)c * Mp);
#pragma unroll
            for (int i = 0; i < RPT / 2; i++) {
                const double2 a = a2[i];
                acc[2 * i] = fma(a.x, xv, acc[2 * i]);
                acc[2 * i + 1] = fma(a.y, xv, acc[2 * i + 1]);
            }
        }
        if (t < nt) {
            const int64_t e = e0 + t;
            const int r0 = rg * RPT;
            if (MODE == 0) {
                double *dst = A.uup + (size_t)A.ent_node[eoff + e] * Q + r0;
#pragma unroll
                for (int i = 0; i < RPT; i++)
                    if (r0 + i < M) dst[i] = acc[i];
            } else if (!(A.ent[eoff + e] & 1)) {
                double *dst = A.udown + (size_t)(A.T.off[l + 1] + 4 * e) * Q + r0;
#pragma unroll
                for (int i = 0; i < RPT; i++)
                    if (r0 + i < M) dst[i] += acc[i];
            }
        }
    }
}

// The same products on the FP64 tensor path (mma.sync m8n8k4 .f64; the FP64
// vector pipe sustains a quarter of its rate).  A block takes 32 entries.  It
// stages by bulk asynchronous copies on one mbarrier: the operator [K][M] row
// by row into a row stride ldo = 4 mod 16 doubles (conflict-free fragment
// loads), the entries' columns X into rows of stride ldx, and for L2L the
// children groups' current u_down (M = 4Q contiguous doubles per entry) into
// C.  Warp w computes all M rows for entries 8w..8w+7 in chunks of 8*MT rows
// (MT 8x8 accumulator tiles); results are written (M2M) or added (L2L) into C
// in shared memory and leave by bulk stores, one row per entry.  Fragments:
// A[row = lane/4][k = lane%4], B[k = lane%4][n = lane/4],
// C[row = lane/4][n = 2*(lane%4) + {0,1}].  Needs M % 8 == 0, K % 4 == 0 and
// 16-byte aligned operator rows.  A copy wait that runs out sets *err and the
// block leaves without writing.
constexpr int LM_THREADS = 128;
static size_t lvl_mma_smem(int M, int K) {
    return ((size_t)K * pad4mod16(M) + 32 * (size_t)pad4mod16(K) + 32 * (size_t)M) * sizeof(double);
}

template <int MODE, int MT>
__global__ void __launch_bounds__(LM_THREADS) k_lvl_mma(PassArgs A, int l, int M, int K, long long wait_limit,
                                                       unsigned long long *err) {
    extern __shared__ __align__(128) double sm_m[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int snode[32];  // node of the entry (M2M), or of a split entry (L2L); -1 otherwise
    const int ldo = pad4mod16(M), ldx = pad4mod16(K), Q = A.Q, tid = threadIdx.x;
    double *opS = sm_m;                  // [K][ldo]
    double *xS = opS + (size_t)K * ldo;  // [32][ldx]
    double *cS = xS + (size_t)32 * ldx;  // [32][M]
    const int64_t ne = A.T.ne[l], eoff = A.T.eoff[l], e0 = (int64_t)blockIdx.x * 32;
    const int nt = (int)min((int64_t)32, ne - e0);
    const double *op = A.ops + (size_t)l * A.stride + (MODE == 0 ? A.off_m2m : A.off_l2l);  // [K][M]
    const size_t child0 = (size_t)A.T.off[l + 1] + 4 * (size_t)e0;  // first child of the block's first entry
    int has = 0;
    if (tid < 32) {
        int node = -1;
        if (tid < nt) {
            const int64_t e = eoff + e0 + tid;
            if (MODE == 0 || !(A.ent[e] & 1)) node = A.ent_node[e];
        }
        snode[tid] = node;
        has = node >= 0;
    }
    const uint32_t mb = smem_u32(&bar);
    if (tid == 0) mbar_init(mb);
    const int nact = __syncthreads_count(has);
    if (tid == 0) mbar_expect_tx(mb, (uint32_t)(K * M + nact * K + (MODE == 1 ? nact * M : 0)) * 8u);
    __syncthreads();
    // the operator does not depend on the previous level: copy it before waiting
    for (int c = tid; c < K; c += LM_THREADS)
        bulk_g2s(smem_u32(opS + (size_t)c * ldo), op + (size_t)c * M, (uint32_t)M * 8u, mb);
    // launched with programmatic stream serialisation: let the next level's
    // kernel be scheduled, then wait until the previous kernel has completed
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    for (int c = K + tid; c < K + 64; c += LM_THREADS) {
        if (c < K + 32) {
            const int n = c - K;
            if (n < nt && snode[n] >= 0) {
                const double *src = MODE == 0 ? A.uup + (child0 + 4 * (size_t)n) * Q : A.udown + (size_t)snode[n] * Q;
                bulk_g2s(smem_u32(xS + (size_t)n * ldx), src, (uint32_t)K * 8u, mb);
            }
        } else if (MODE == 1) {
            const int n = c - K - 32;
            if (n < nt && snode[n] >= 0)
                bulk_g2s(smem_u32(cS + (size_t)n * M), A.udown + (child0 + 4 * (size_t)n) * Q, (uint32_t)M * 8u, mb);
        }
    }
    const bool ok = __syncthreads_and(mbar_wait(mb, 0, wait_limit));
    if (!ok) {
        if (tid == 0) atomicOr(err, 1ull);
        mbar_wait(mb, 0, kDrainWaitPolls);  // let copies in flight land before the block leaves
        return;
    }
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    const int n0 = warp * 8;
    if (n0 < nt) {
        const double *xb = xS + (size_t)(n0 + g) * ldx + t;
        for (int rc = 0; rc < M; rc += 8 * MT) {
            double acc[MT][2];
#pragma unroll
            for (int i = 0; i < MT; i++) acc[i][0] = acc[i][1] = 0.0;
            const double *ab = opS + (size_t)t * ldo + rc + g;
#pragma unroll 2
            for (int k0 = 0; k0 < K; k0 += 4) {
                const double b = xb[k0];
#pragma unroll
                for (int i = 0; i < MT; i++)
                    if (rc + 8 * i < M) dmma_8x8x4(acc[i][0], acc[i][1], ab[(size_t)k0 * ldo + 8 * i], b);
            }
#pragma unroll
            for (int i = 0; i < MT; i++) {
                const int r = rc + 8 * i + g;
                if (r >= M) continue;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int n = n0 + 2 * t + j;
                    if (n >= nt || snode[n] < 0) continue;
                    if (MODE == 0) cS[(size_t)n * M + r] = acc[i][j];
                    else cS[(size_t)n * M + r] += acc[i][j];
                }
            }
        }
    }
    fence_proxy_async();
    __syncthreads();
    if (tid < nt && snode[tid] >= 0) {
        double *dst = MODE == 0 ? A.uup + (size_t)snode[tid] * Q : A.udown + (child0 + 4 * (size_t)tid) * Q;
        bulk_s2g(dst, smem_u32(cS + (size_t)tid * M), (uint32_t)M * 8u);
        bulk_commit();
        bulk_wait_read();
    }
}

template <int MODE, int MT>
static void launch_lvl_mma(kifmm_plan *P, const PassArgs &A, int l, int M, int K, size_t smem) {
    ensure_dyn_smem(k_lvl_mma<MODE, MT>, smem);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((P->lt.ne[l] + 31) / 32));
    cfg.blockDim = dim3(LM_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = P->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // overlap with the previous level's tail
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    KIFMM_CUDA(cudaLaunchKernelEx(&cfg, k_lvl_mma<MODE, MT>, A, l, M, K, plan_wait_polls(P),
                                  P->scal.p + KIFMM_SCAL_PASS_ERR));
    KIFMM_LAUNCHED();
}

// NT columns per block: (ceil(M/4)) x (NT/4) threads <= 256 and at most
// 200 KB of shared memory
static int lvl_gemm_nt(int M, int K) {
    int tm = (M + 3) / 4;
    int nt = (256 / tm) * 4;
    if (nt > 32) nt = 32;  // more blocks per level: the levels are small
    int cap = (int)(((200 << 10) / 8 - (int64_t)K * M) / (K + 1)) / 4 * 4;
    if (nt > cap) nt = cap;
    return nt < 4 ? 4 : nt;
}

template <int MODE>
static void launch_lvl_gemm(kifmm_plan *P, const PassArgs &A, int l) {
    const int Q = P->Q;
    const int M = MODE == 0 ? Q : 4 * Q, K = MODE == 0 ? 4 * Q : Q;
    const int64_t ne = P->lt.ne[l];
    if (M % 8 == 0 && K % 4 == 0 && A.stride % 2 == 0 && A.off_m2m % 2 == 0 && A.off_l2l % 2 == 0) {
        // FP64 tensor path with bulk-copy staging (16-byte aligned rows)
        const size_t smem = lvl_mma_smem(M, K);
        if (smem <= (size_t)(220 << 10)) {
            const int mt = M / 8;
            if (mt <= 2) launch_lvl_mma<MODE, 2>(P, A, l, M, K, smem);
            else if (mt <= 4) launch_lvl_mma<MODE, 4>(P, A, l, M, K, smem);
            else if (mt <= 8) launch_lvl_mma<MODE, 8>(P, A, l, M, K, smem);
            else launch_lvl_mma<MODE, 16>(P, A, l, M, K, smem);
            return;
        }
    }
    {  // broadcast form when the operator and the entry tile fit in shared memory
        constexpr int RPT = MODE == 0 ? 8 : 16;
        const int RG = (M + RPT - 1) / RPT, Mp = RG * RPT;
        const int wps = RG < 8 ? RG : 8, NT = 32 * (8 / wps);
        const size_t smem = ((size_t)K * Mp + (size_t)NT * (K + 1)) * sizeof(double);
        if (smem <= (size_t)(220 << 10)) {
            ensure_dyn_smem(k_lvl_gemm_b<MODE, RPT>, smem);
            k_lvl_gemm_b<MODE, RPT><<<(unsigned)((ne + NT - 1) / NT), LG_THREADS, smem, P->stream>>>(A, l, M, K, Mp,
                                                                                                     NT);
            KIFMM_LAUNCHED();
            return;
        }
    }
    int nt = lvl_gemm_nt(M, K);
    int threads = ((M + 3) / 4) * (nt / 4);
    size_t smem = ((size_t)K * M + (size_t)nt * (K + 1)) * sizeof(double);
    ensure_dyn_smem(k_lvl_gemm_d<MODE>, smem);
    k_lvl_gemm_d<MODE><<<(unsigned)((ne + nt - 1) / nt), threads, smem, P->stream>>>(A, l, M, K, nt);
    KIFMM_LAUNCHED();
}

void launch_m2m_d(kifmm_plan *P, const PassArgs &A, int l) { launch_lvl_gemm<0>(P, A, l); }
void launch_l2l_d(kifmm_plan *P, const PassArgs &A, int l) { launch_lvl_gemm<1>(P, A, l); }

// the upward M2M over levels L-2 .. 2 and the downward L2L over 2 .. L-2
void run_m2m_levels(kifmm_plan *P, const PassArgs &A) {
    for (int l = P->L - 2; l >= 2; l--)
        if (P->lt.ne[l]) launch_m2m_d(P, A, l);
}
void run_l2l_levels(kifmm_plan *P, const PassArgs &A) {
    for (int l = 2; l <= P->L - 2; l++)
        if (P->lt.ne[l]) launch_l2l_d(P, A, l);
}

// Buffers of an apply, its cleared flags and expansions, and the densities in
// tree order.
void apply_prologue(kifmm_plan *P) {
    cudaStream_t s = P->stream;
    const int Q = P->Q;
    int64_t n = P->N, NN = P->n_nodes;
    const int64_t vw = P->cplx ? 2 : 1;  // doubles per density value
    P->taus.alloc(n * vw);
    P->pots.alloc(n * vw);
    P->uup.alloc((size_t)NN * Q);
    P->udown.alloc((size_t)NN * Q);
    // error flags of the level passes and the tensor-core M2L, and the
    // expansions, cleared first so that the kernels below form one chain of
    // programmatic dependent launches
    KIFMM_CUDA(cudaMemsetAsync(P->scal.p + KIFMM_SCAL_PASS_ERR, 0,
                               (KIFMM_SCAL_WORDS - KIFMM_SCAL_PASS_ERR) * sizeof(unsigned long long), s));
    KIFMM_CUDA(cudaMemsetAsync(P->uup.p, 0, (size_t)NN * Q * sizeof(double), s));
    KIFMM_CUDA(cudaMemsetAsync(P->udown.p, 0, (size_t)NN * Q * sizeof(double), s));
    if (P->opt.planned) {
        ops_wait_now(P);
        build_plan_matrices(P);  // first apply after build_tree / precompute
    }
    ops_wait_circles(P);  // the P2M's check points
    if (P->cplx)
        launch_gather_tau_c(P);
    else
        launch_pdl(k_gather_tau, dim3(grid_for(n, 256, P->num_sms * 8)), dim3(256), 0, s, (const double *)P->tau.p,
                   (const int32_t *)P->perm.p, n, P->taus.p);
}

void run_upward_downward(kifmm_plan *P) {
    cudaStream_t s = P->stream;
    const int Q = P->Q, L = P->L;
    near_join(P);  // the previous apply's near-field pass, if never evaluated
    apply_prologue(P);
    if (P->opt.precision == KIFMM_PREC_MIXED) {
        run_passes_mixed(P);
        ops_wait_now(P);  // (L < 3: the evaluation reads them)
        return;
    }
    if (L < 3) {  // no level has well-separated boxes
        ops_wait_now(P);
        return;
    }
    PassArgs A = make_pass_args(P);
    if (P->n_p2m_list) {
        PhaseScope ph(P, KIFMM_PHASE_P2M);
        if (P->cplx) launch_p2m_c(P, A);
        else if (planned_ready(P)) launch_planned_p2m(P, A);
        else launch_p2m_d(P, A);
    }
    ops_wait_now(P);  // the P2M reads only the check circles
    {
        PhaseScope ph_m2m(P, KIFMM_PHASE_M2M);
        run_m2m_levels(P, A);
    }
    if (Q % 2 == 0 && 4 * Q <= 8 * MD_MT * 8) {
        // FP64 tensor path: all levels' M2L in one launch, then the L2L chain
        M2lDmmaArgs M{};
        M.A = A;
        if (!P->zero4q.p) {
            P->zero4q.alloc((size_t)4 * Q);
            KIFMM_CUDA(cudaMemsetAsync(P->zero4q.p, 0, (size_t)4 * Q * sizeof(double), s));
        }
        M.zero = P->zero4q.p;
        M.lmin = 1;
        M.lmax = L - 2;
        M.wait_limit = plan_wait_polls(P);
        M.err = P->scal.p + KIFMM_SCAL_PASS_ERR;
        int64_t tiles = 0;
        for (int l = 0; l <= MAX_LEVELS; l++) {
            M.tile_off[l] = tiles;
            if (l >= M.lmin && l <= M.lmax) tiles += (P->lt.ne[l] + MD_TE - 1) / MD_TE;
        }
        {
            PhaseScope ph(P, KIFMM_PHASE_M2L);
            if (tiles) {
                const size_t smem = m2l_dmma_smem(4 * Q);
                ensure_dyn_smem(k_m2l_dmma, smem);
                launch_pdl(k_m2l_dmma, dim3((unsigned)tiles), dim3(MD_BLOCK), smem, s, M);
            }
        }
        PhaseScope ph(P, KIFMM_PHASE_L2L);
        run_l2l_levels(P, A);
        return;
    }
    PhaseScope ph(P, KIFMM_PHASE_M2L);
    int thr = ((4 * Q + 31) / 32) * 32;
    size_t smem = (size_t)M2L_TE * 4 * Q * sizeof(double);
    ensure_dyn_smem(k_m2l_d, smem);
    for (int l = 1; l <= L - 2; l++) {
        int64_t ne = P->lt.ne[l];
        if (!ne) continue;
        k_m2l_d<<<(unsigned)((ne + M2L_TE - 1) / M2L_TE), thr, smem, s>>>(A, l);
        KIFMM_LAUNCHED();
    }
}

// potentials from tree order to the caller's order
void launch_scatter_pot(kifmm_plan *P) {
    const int64_t n = P->N;
    launch_pdl(k_scatter_pot, dim3(grid_for(n, 256, P->num_sms * 8)), dim3(256), 0, P->stream,
               (const double *)P->pots.p, (const int32_t *)P->perm.p, n, P->pot_out.p);
}

void run_eval_sources(kifmm_plan *P, int check_self) {
    int64_t n = P->N;
    P->pot_out.alloc(P->cplx ? 2 * n : n);
    if (P->cplx) {
        run_eval_sources_c(P, make_pass_args(P), check_self);
        return;
    }
    if (check_self && planned_ready(P)) {
        if (P->n_leaf_list) {
            PhaseScope ph(P, KIFMM_PHASE_LEAF);
            launch_planned_leaf(P, make_pass_args(P));
        }
    } else if (P->opt.precision == KIFMM_PREC_MIXED) {
        run_eval_sources_mixed(P, check_self);
    } else {
        PassArgs A = make_pass_args(P);
        if (P->n_leaf_list) {
            PhaseScope ph(P, KIFMM_PHASE_LEAF);
            launch_leaf_eval_d(P, A, check_self);
        }
    }
    launch_scatter_pot(P);
}

void run_eval_targets(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self, double *pot) {
    PassArgs A = make_pass_args(P);
    if (P->cplx) {
        run_eval_targets_c(P, A, tx, ty, n, check_self, pot);
        return;
    }
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

void direct_sum_device_c(const kifmm_kernel &kn, const double *x, const double *y, const double *tau, int64_t n,
                         const int64_t *tg, int64_t nt, double *out, cudaStream_t s);
void kernel_matrix_device_c(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                            const double *ty, int64_t nt, double *out, cudaStream_t s);
void kernel_apply_device_c(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                           const double *ty, int64_t nt, const double *tau, double *out, cudaStream_t s);

void direct_sum_device(const kifmm_kernel &kn, const double *x, const double *y, const double *tau, int64_t n,
                       const int64_t *tg, int64_t nt, double *out, cudaStream_t s) {
    if (kn.kind == KIFMM_KERNEL_HELMHOLTZ) return direct_sum_device_c(kn, x, y, tau, n, tg, nt, out, s);
    if (nt <= 0) return;
    KIFMM_REQUIRE(nt < (1ll << 31), KIFMM_ERR_ARG, "direct_sum: too many targets");
    k_direct_d<<<(unsigned)nt, 256, 0, s>>>(kn.kind, kn.k, x, y, tau, n, tg, out);
    KIFMM_LAUNCHED();
}

void kernel_matrix_device(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                          const double *ty, int64_t nt, double *out, cudaStream_t s) {
    if (kn.kind == KIFMM_KERNEL_HELMHOLTZ) return kernel_matrix_device_c(kn, sx, sy, ns, tx, ty, nt, out, s);
    if (ns * nt <= 0) return;
    k_kmatrix_d<<<grid_for(ns * nt, 256, 8192), 256, 0, s>>>(kn.kind, kn.k, sx, sy, ns, tx, ty, nt, out);
    KIFMM_LAUNCHED();
}

void kernel_apply_device(const kifmm_kernel &kn, const double *sx, const double *sy, int64_t ns, const double *tx,
                         const double *ty, int64_t nt, const double *tau, double *out, cudaStream_t s) {
    if (kn.kind == KIFMM_KERNEL_HELMHOLTZ) return kernel_apply_device_c(kn, sx, sy, ns, tx, ty, nt, tau, out, s);
    if (nt <= 0) return;
    k_kapply_d<<<grid_for(nt, 128, 8192), 128, 0, s>>>(kn.kind, kn.k, sx, sy, ns, tx, ty, nt, tau, out);
    KIFMM_LAUNCHED();
}

}  // namespace kifmm
