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
// Coincident source/target pairs contribute zero, as in the reference.
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
                const int je = m2l_source_entry(A.ncoll, A.nent, A.nbot, A.ntop, p, d);
                if (je >= 0) grp = A.T.off[l + 1] + 4 * (je - A.T.eoff[l]);
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

// Taylor coefficients of every leaf's local expansion (Laplace, levels >= 2),
// FP64 on the tensor path: C[R x leaves] = Taylor_l[R x Q] . u_down[Q x leaves],
// one block per 32 consecutive leaves of one level (leaf_list is level-major).
// Warp w computes all R rows (MTR 8-row tiles) for leaves 8w..8w+7; the block
// writes its 32 x R coefficients as one contiguous run.
struct TaylorArgs {
    PassArgs A;
    const int32_t *list;
    double *coef;
    int lmin, lmax;
    int64_t loff[MAX_LEVELS + 1];  // leaf_list range of each level
    int64_t toff[MAX_LEVELS + 1];  // first block of each level
};
constexpr int TY_THREADS = 128;
constexpr int TY_R = 2 * KIFMM_TAYLOR_P + 1, TY_MTR = (TY_R + 7) / 8;
__global__ void __launch_bounds__(TY_THREADS) k_leaf_taylor(TaylorArgs T) {
    extern __shared__ __align__(16) double sm_ty[];
    const PassArgs &A = T.A;
    const int Q = A.Q, R = TY_R, ldt = pad4mod16(8 * TY_MTR), ldx = pad4mod16(Q);
    double *tS = sm_ty;                      // [Q][ldt]: element (row r, col k) at k * ldt + r
    double *xS = tS + (size_t)Q * ldt;       // [32 leaves][ldx]
    double *cS = xS + 32 * (size_t)ldx;      // [32 leaves][R]
    pdl_trigger();
    const int64_t b = blockIdx.x;
    int l = T.lmin;
    while (l < T.lmax && T.toff[l + 1] <= b) l++;
    const int64_t w0 = T.loff[l] + (b - T.toff[l]) * 32;
    const int nt = (int)min((int64_t)32, T.loff[l + 1] - w0);
    const int tid = threadIdx.x;
    // the level's map (precomputed, independent of the previous kernel), rows padded with zeros
    const double *tl = A.taylor + (size_t)l * Q * R;
    for (int i0 = tid; i0 < Q * ldt; i0 += 4 * TY_THREADS) {
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = i0 + q * TY_THREADS, k = i / ldt, r = i - k * ldt;
            v[q] = (i < Q * ldt && r < R) ? tl[(size_t)k * R + r] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = i0 + q * TY_THREADS;
            if (i < Q * ldt) tS[i] = v[q];
        }
    }
    pdl_wait();  // u_down comes from the L2L chain
    for (int i0 = tid; i0 < 32 * Q; i0 += 4 * TY_THREADS) {
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = i0 + q * TY_THREADS, n = i / Q, k = i - n * Q;
            v[q] = (i < 32 * Q && n < nt) ? A.udown[(size_t)T.list[w0 + n] * Q + k] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = i0 + q * TY_THREADS, n = i / Q, k = i - n * Q;
            if (i < 32 * Q) xS[n * ldx + k] = v[q];
        }
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3, n0 = warp * 8;
    if (n0 < nt) {
        double acc[TY_MTR][2];
#pragma unroll
        for (int i = 0; i < TY_MTR; i++) acc[i][0] = acc[i][1] = 0.0;
        const double *xb = xS + (size_t)(n0 + g) * ldx + t;
        const double *ab = tS + (size_t)t * ldt + g;
        for (int k0 = 0; k0 < Q; k0 += 4) {
            const double bv = xb[k0];
#pragma unroll
            for (int i = 0; i < TY_MTR; i++) dmma_8x8x4(acc[i][0], acc[i][1], ab[(size_t)k0 * ldt + 8 * i], bv);
        }
#pragma unroll
        for (int i = 0; i < TY_MTR; i++) {
            const int r = 8 * i + g;
            if (r < R) {
                cS[(n0 + 2 * t) * R + r] = acc[i][0];
                cS[(n0 + 2 * t + 1) * R + r] = acc[i][1];
            }
        }
    }
    __syncthreads();
    double *out = T.coef + (size_t)w0 * R;
    for (int i = tid; i < nt * R; i += TY_THREADS) out[i] = cS[i];
}

// L2P + P2P: one warp per target leaf.  The sources of the leaf and its eight
// colleagues are staged in shared memory as one list (the leaf's own points
// first), in chunks of LEAF_CHUNK.  A tile of nt <= 32 targets is spread over
// the warp in ng groups (two targets per lane for the Laplace kernel, one
// otherwise) with sp = 32 / ng lanes per group, each lane taking every sp-th
// source, so a leaf of 15 points keeps 32 lanes busy and no lane idles on a
// short colleague; the Laplace pair loop runs on packed FP32 pairs (f32x2),
// one instruction for both of a lane's targets.  For the Laplace kernel the
// offsets are scaled by 1/w (w the leaf width) so every log2 term is O(1); the
// remainder log2(w^2) * sum(tau) is added in FP64.  The inner loop is
// branch-free: r^2 is floored at FLT_MIN (r^2 + FLT_MIN) and short chunks are
// padded with far, uncharged sources.  The pairs inside the leaf itself that
// meet the floor (the target's own point and exact duplicates, which the
// reference skips, class_fmm.py:107) are counted in the first passes, over
// the leaf's own points, and taken back out.  Distinct points of different
// leaves closer than about 2^-24 leaf widths round to the same FP32 offsets
// and keep log2(FLT_MIN) for their pair; the FP64 near field (near_fp64)
// resolves such pairs.  FP32 partial sums of at most 32 terms are accumulated
// in FP64.
// one warp per block: leaves differ in work by more than 10x, and a block of
// several warps would hold its SM slot until its slowest warp is done
constexpr int LEAF_WARPS = 1;
// 32 one-warp blocks per SM (64 registers) with 96-source chunks measured 2%
// faster than 28 blocks (72 registers) with 128-source chunks on the 1M
// mixture (0.240 against 0.244 ms), and those 8% faster than 20 blocks (96
// registers) with 256-source chunks; shared memory per block sets the ceiling
#ifndef KIFMM_LEAF_BLOCKS_PER_SM
#define KIFMM_LEAF_BLOCKS_PER_SM 32
#endif
#ifndef KIFMM_LEAF_CHUNK
#define KIFMM_LEAF_CHUNK 96
#endif
constexpr int LEAF_BLOCKS_PER_SM = KIFMM_LEAF_BLOCKS_PER_SM;  // resident blocks per SM at the register bound
constexpr int LEAF_CHUNK = KIFMM_LEAF_CHUNK;                  // sources staged per pass
static_assert(LEAF_CHUNK + 31 <= 200, "the leaf kernel's quotients (small_div) need cn + sp - 1 <= 200");

__device__ __forceinline__ float lg2_ftz(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float pair_r2(float tx, float ty, const float4 &sv) {
    const float dx = tx - sv.x, dy = ty - sv.y;
    return fmaf(dx, dx, dy * dy);
}
// log2 of r^2 + FLT_MIN: the floor rides in the r^2 multiply-add instead of
// a separate clamp.  Every pair of distinct points has r^2 >= 2^-48 (scaled
// FP32 offsets of O(1)), where adding 2^-126 changes nothing; coincident
// points give log2(FLT_MIN) exactly, as the clamp does.
__device__ __forceinline__ float pair_lg2_floor(float tx, float ty, const float4 &sv) {
    const float dx = tx - sv.x, dy = ty - sv.y;
    return lg2_ftz(fmaf(dx, dx, fmaf(dy, dy, 1.17549435e-38f)));
}

// Packed FP32 pairs (sm_100 .f32x2 arithmetic): one 64-bit register holds a
// value for each of a lane's two targets.  Sources are staged with their
// coordinates and charge duplicated, (x, x | y, y) and (z, z), so one
// instruction forms both targets' offsets, squared distances and products:
// the same IEEE operations as the scalar form, issued half as often.
typedef unsigned long long f32x2;
constexpr f32x2 F2_FLOOR = 0x0080000000800000ull;  // (FLT_MIN, FLT_MIN)
__device__ __forceinline__ f32x2 f2_pack(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// r^2 + FLT_MIN of both targets to one source (as pair_lg2_floor)
__device__ __forceinline__ f32x2 pair2_r2_floor(f32x2 tx, f32x2 ty, const ulonglong2 &s) {
    const f32x2 dx = f2_sub(tx, s.x), dy = f2_sub(ty, s.y);
    return f2_fma(dx, dx, f2_fma(dy, dy, F2_FLOOR));
}
__device__ __forceinline__ f32x2 lg2_pair(f32x2 r) {
    float a, b;
    f2_unpack(r, a, b);
    return f2_pack(lg2_ftz(a), lg2_ftz(b));
}

// Laplace pair sums of one lane holding two targets (tx, ty packed): over its
// sources at list positions j + k SP, k in [k0, k1), of z log2(r^2 + FLT_MIN),
// in FP32 blocks of at most 32 sources (two chains per target, alternating
// sources) added to na, nb in FP64.  OWN: the positions are the leaf's own
// points below en, where coincident pairs (the target itself, duplicates) meet
// the floor; their charges are summed into exa, exb to be taken out.  SP is a
// template argument so that the strided shared-memory loads take immediate
// offsets.
template <int SP_, bool OWN>
__device__ __forceinline__ void leaf_pairs2(const ulonglong2 *__restrict__ sxy, const f32x2 *__restrict__ sz, int j,
                                            int k0, int k1, f32x2 tx, f32x2 ty, int en, double &na, double &nb,
                                            float &exa, float &exb, int sp_rt = 0) {
    constexpr float FLOOR2 = 2.0f * 1.17549435e-38f;
    const int SP = SP_ ? SP_ : sp_rt;
    for (int kb = k0; kb < k1; kb += 32) {
        const int ke = min(k1, kb + 32);
        f32x2 acc0 = 0ull, acc1 = 0ull;
        const ulonglong2 *p = sxy + j + kb * SP;
        const f32x2 *q = sz + j + kb * SP;
        int k = kb;
        if (OWN) {
            for (; k < ke; k++, p += SP, q += SP) {
                const f32x2 r = pair2_r2_floor(tx, ty, *p), z = *q;
                acc0 = f2_fma(z, lg2_pair(r), acc0);
                float ra, rb, zs, zu;
                f2_unpack(r, ra, rb);
                f2_unpack(z, zs, zu);
                const bool in = j + k * SP < en;
                exa += (in && ra < FLOOR2) ? zs : 0.f;
                exb += (in && rb < FLOOR2) ? zs : 0.f;
            }
        } else {
#pragma unroll 1
            for (; k + 3 < ke; k += 4, p += 4 * SP, q += 4 * SP) {
                const ulonglong2 s0 = p[0], s1 = p[SP], s2 = p[2 * SP], s3 = p[3 * SP];
                const f32x2 z0 = q[0], z1 = q[SP], z2 = q[2 * SP], z3 = q[3 * SP];
                acc0 = f2_fma(z0, lg2_pair(pair2_r2_floor(tx, ty, s0)), acc0);
                acc1 = f2_fma(z1, lg2_pair(pair2_r2_floor(tx, ty, s1)), acc1);
                acc0 = f2_fma(z2, lg2_pair(pair2_r2_floor(tx, ty, s2)), acc0);
                acc1 = f2_fma(z3, lg2_pair(pair2_r2_floor(tx, ty, s3)), acc1);
            }
            for (; k + 1 < ke; k += 2, p += 2 * SP, q += 2 * SP) {
                acc0 = f2_fma(q[0], lg2_pair(pair2_r2_floor(tx, ty, p[0])), acc0);
                acc1 = f2_fma(q[SP], lg2_pair(pair2_r2_floor(tx, ty, p[SP])), acc1);
            }
            if (k < ke) acc0 = f2_fma(q[0], lg2_pair(pair2_r2_floor(tx, ty, p[0])), acc0);
        }
        float sa, sb;
        f2_unpack(f2_add(acc0, acc1), sa, sb);
        na += (double)sa;
        nb += (double)sb;
    }
}
// leaf_pairs2 for a run-time lane stride sp = 32 / groups, groups in 1..16
template <bool OWN>
__device__ __forceinline__ void leaf_pairs2_sp(int sp, const ulonglong2 *sxy, const f32x2 *sz, int j, int k0, int k1,
                                               f32x2 tx, f32x2 ty, int en, double &na, double &nb, float &exa,
                                               float &exb) {
#define KIFMM_LEAF_SP(S)                                                          \
    case S:                                                                       \
        leaf_pairs2<S, OWN>(sxy, sz, j, k0, k1, tx, ty, en, na, nb, exa, exb); \
        break;
#ifndef KIFMM_LEAF_SP_MODE
#define KIFMM_LEAF_SP_MODE 1
#endif
#if KIFMM_LEAF_SP_MODE == 0
    leaf_pairs2<0, OWN>(sxy, sz, j, k0, k1, tx, ty, en, na, nb, exa, exb, sp);
#elif KIFMM_LEAF_SP_MODE == 1
    if (sp == 2) leaf_pairs2<2, OWN>(sxy, sz, j, k0, k1, tx, ty, en, na, nb, exa, exb);
    else leaf_pairs2<0, OWN>(sxy, sz, j, k0, k1, tx, ty, en, na, nb, exa, exb, sp);
#else
    switch (sp) {
        KIFMM_LEAF_SP(2)
        KIFMM_LEAF_SP(3)
        KIFMM_LEAF_SP(4)
        KIFMM_LEAF_SP(5)
        KIFMM_LEAF_SP(6)
        KIFMM_LEAF_SP(8)
        KIFMM_LEAF_SP(10)
        KIFMM_LEAF_SP(16)
        default:
            leaf_pairs2<32, OWN>(sxy, sz, j, k0, k1, tx, ty, en, na, nb, exa, exb);
    }
#endif
#undef KIFMM_LEAF_SP
}

// x / d for 0 <= x <= 200 and 1 <= d <= 32 as a multiply and a shift (the
// lane-layout quotients of the leaf kernel; a division by a run-time value
// costs a reciprocal and a dozen fix-up instructions): c = ceil(2^16 / d)
// gives floor(x c / 2^16) = floor(x / d) whenever x < 2^16 / d.
__constant__ unsigned c_recip16[33] = {
    0,    65536, 32768, 21846, 16384, 13108, 10923, 9363, 8192, 7282, 6554, 5958, 5462, 5042, 4682, 4370, 4096,
    3856, 3641,  3450,  3277,  3121,  2979,  2850,  2731, 2622, 2521, 2428, 2341, 2260, 2185, 2115, 2048};
__device__ __forceinline__ int small_div(int x, int d) { return (int)(((unsigned)x * c_recip16[d]) >> 16); }

// the L2P + P2P of leaf w of A's leaf list, by one warp: its 32-target tiles
// [tile0, tile1) (all of them by default).  PART: LEAF_BOTH writes near + far
// field, LEAF_NEAR the near field alone (P2P, run under the far-field chain),
// LEAF_FAR adds the far field (L2P) to what LEAF_NEAR wrote.
enum LeafPart { LEAF_BOTH = 0, LEAF_NEAR = 1, LEAF_FAR = 2 };
template <int KIND, int PART = LEAF_BOTH>
__device__ __forceinline__ void leaf_eval_f_leaf(const PassArgs &A, int64_t w, int tile0 = 0, int tile1 = 1 << 20) {
    constexpr int R = 2 * KIFMM_TAYLOR_P + 1;
    constexpr float CLAMP = 1.17549435e-38f;  // FLT_MIN
    __shared__ ulonglong2 sxys[LEAF_WARPS][LEAF_CHUNK + 32];  // (x, x | y, y) per staged source
    __shared__ f32x2 szs[LEAF_WARPS][LEAF_CHUNK + 32];        // (z, z)
    __shared__ double qds[LEAF_WARPS][R > 64 ? R : 64];
    __shared__ float qfs[LEAF_WARPS][R > 64 ? R : 64];
    __shared__ double red[LEAF_WARPS][2][32];
    __shared__ float redf[LEAF_WARPS][2][32];
    __shared__ int rngs[LEAF_WARPS][18];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    {
        // the leaf record: node, level, point range, cell key and source ranges
        // in one coalesced load (list[w] is the record's node)
        const int rv = A.leaf_rec[w * LEAF_REC_WORDS + lane];
        const int g = __shfl_sync(0xffffffffu, rv, LR_NODE);
        const int l = __shfl_sync(0xffffffffu, rv, LR_LEVEL);
        const uint64_t key = (uint64_t)(uint32_t)__shfl_sync(0xffffffffu, rv, LR_KEY_LO) |
                             ((uint64_t)(uint32_t)__shfl_sync(0xffffffffu, rv, LR_KEY_HI) << 32);
        double cx, cy;
        {
            const double wl = ldexp(A.W, -l);
            cx = A.root + ((double)compact2(key >> 1) + 0.5) * wl;
            cy = A.root + ((double)compact2(key) + 0.5) * wl;
        }
        const bool lap = KIND == KIFMM_KERNEL_LAPLACE;
        const bool taylor = lap && A.taylor != nullptr && l >= 2 && PART != LEAF_NEAR;
        double *qd = qds[wib];
        float *qf = qfs[wib];
        ulonglong2 *sxy = sxys[wib];
        f32x2 *sz = szs[wib];
        const double width = ldexp(A.W, -l);
        const double sc = lap ? 1.0 / width : 1.0;     // coordinate scale
        const double lw = lap ? -2.0 * log2(sc) : 0.0; // log2 of the squared length unit
        if (taylor) {  // Taylor coefficients of the local expansion (k_leaf_taylor, FP64)
            const double *cf = A.leaf_coef + (size_t)w * R;
            for (int r = lane; r < R; r += 32) {
                const double v = cf[r];
                qd[r] = v;
                qf[r] = (float)v;
            }
        } else if (PART != LEAF_NEAR) {
            local_density(A, g, l, qd, lane);
        }
        const float kk = (float)A.k;
        const float lclamp = lg2_ftz(CLAMP);
        const int b = __shfl_sync(0xffffffffu, rv, LR_BOT), e = __shfl_sync(0xffffffffu, rv, LR_TOP);
        const int ns = __shfl_sync(0xffffffffu, rv, LR_NSRC);
        // source ranges: the leaf itself, then its colleagues in direction order;
        // list element p lies in the last range i with pre[i] <= p, at p + off[i]
        // (kept in shared memory: registers are scarce in the pair loop)
        int *rng = rngs[wib];
        if (lane >= LR_RNG && lane < LR_RNG + 18) rng[lane - LR_RNG] = rv;
        double tsum = 0.0;  // FP64 sum of the near sources' charges (Laplace)
        // stage sources [c0, c0 + cn) of the list, padded with 32 far, uncharged
        // ones; four elements per lane per pass, loads issued before any is used
        auto gather = [&](int c0, int cn, bool sum) {
            __syncwarp();
            int pre[9], off[9];
    #pragma unroll
            for (int i = 0; i < 9; i++) {
                pre[i] = rng[i];
                off[i] = rng[9 + i];
            }
            for (int q0 = 0; q0 < cn; q0 += 128) {
                int si[4];
    #pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int q = q0 + lane + 32 * k, p = c0 + q;
                    int sv = p + off[0];
    #pragma unroll
                    for (int i = 1; i < 9; i++) sv = p >= pre[i] ? p + off[i] : sv;
                    si[k] = q < cn ? sv : -1;
                }
                double vx[4], vy[4], vt[4];
    #pragma unroll
                for (int k = 0; k < 4; k++)
                    if (si[k] >= 0) {
                        vx[k] = A.xs[si[k]];
                        vy[k] = A.ys[si[k]];
                        vt[k] = A.taus[si[k]];
                    }
    #pragma unroll
                for (int k = 0; k < 4; k++)
                    if (si[k] >= 0) {
                        const float fx = (float)((vx[k] - cx) * sc), fy = (float)((vy[k] - cy) * sc);
                        const float fz = (float)vt[k];
                        sxy[q0 + lane + 32 * k] = make_ulonglong2(f2_pack(fx, fx), f2_pack(fy, fy));
                        sz[q0 + lane + 32 * k] = f2_pack(fz, fz);
                        if (sum) tsum += vt[k];
                    }
            }
            sxy[cn + lane] = make_ulonglong2(f2_pack(1e18f, 1e18f), f2_pack(1e18f, 1e18f));
            sz[cn + lane] = 0ull;
            __syncwarp();
        };
        __syncwarp();
        const int tfirst = b + 32 * tile0, tend = (int)min((int64_t)e, (int64_t)b + 32 * (int64_t)tile1);
        for (int t0 = tfirst; t0 < tend; t0 += 32) {
            const int nt = min(32, e - t0);
            // Lane layout: the tile's targets form ng groups of tb targets
            // (two for the Laplace kernel, one otherwise); sp = 32 / ng lanes
            // share a group, lane (gi, j) taking sources j, j + sp, ...  Two
            // targets per lane share each source load and every packed
            // (f32x2) instruction of the pair loop.
            const int ng = lap ? (nt + 1) >> 1 : nt, sp = small_div(32, ng);
            const int j = small_div(lane, ng), gi = lane - j * ng;
            const int ia = gi, ib = lap && gi + ng < nt ? gi + ng : gi;  // second slot repeats the first when unused
            const float txa = (float)((A.xs[t0 + ia] - cx) * sc), tya = (float)((A.ys[t0 + ia] - cy) * sc);
            const float txb = (float)((A.xs[t0 + ib] - cx) * sc), tyb = (float)((A.ys[t0 + ib] - cy) * sc);
            const f32x2 tx2 = f2_pack(txa, txb), ty2 = f2_pack(tya, tyb);
            double neara = 0.0, nearb = 0.0;
            float exa = 0.f, exb = 0.f;  // charges of the leaf's own points met at the floor
            for (int c0 = 0; PART != LEAF_FAR && c0 < ns; c0 += LEAF_CHUNK) {
                const int cn = min(LEAF_CHUNK, ns - c0);
                if (t0 == tfirst || ns > LEAF_CHUNK) gather(c0, cn, lap && t0 == tfirst);
                // lane (gi, j) takes sources j, j + sp, ...; j + (it - 1) sp < cn + 32
                const int it = small_div(cn + sp - 1, sp);
                if (KIND == KIFMM_KERNEL_LAPLACE) {
                    // the list starts with the leaf's own points, local [0, en): the
                    // first kown passes count the pairs there that meet the floor
                    const int en = min(e - b - c0, cn);
                    const int kown = en > 0 ? small_div(en + sp - 1, sp) : 0;
                    leaf_pairs2_sp<true>(sp, sxy, sz, j, 0, kown, tx2, ty2, en, neara, nearb, exa, exb);
                    leaf_pairs2_sp<false>(sp, sxy, sz, j, kown, it, tx2, ty2, en, neara, nearb, exa, exb);
                } else {
                    for (int k0 = 0; k0 < it; k0 += 32) {
                        const int k1 = min(it, k0 + 32);
                        float acc = 0.f;
    #pragma unroll 1
                        for (int k = k0; k < k1; k++) {
                            const int u = j + k * sp;
                            float sx, sy, sw, unused;
                            f2_unpack(sxy[u].x, sx, unused);
                            f2_unpack(sxy[u].y, sy, unused);
                            f2_unpack(sz[u], sw, unused);
                            const float4 sv = make_float4(sx, sy, sw, 0.f);
                            const float r2 = pair_r2(txa, tya, sv);
                            if (r2 > 0.f) acc = fmaf(sv.z, gsum_term<KIND>(r2, kk), acc);
                        }
                        neara += (double)acc;
                    }
                }
            }
            if (lap && t0 == tfirst)
                for (int o = 16; o; o >>= 1) tsum += __shfl_xor_sync(0xffffffffu, tsum, o);
            // per-lane shares with the clamped own pairs taken out
            red[wib][0][lane] = lap ? neara - (double)exa * (double)lclamp : neara;
            red[wib][1][lane] = lap ? nearb - (double)exb * (double)lclamp : nearb;
            redf[wib][0][lane] = exa;
            redf[wib][1][lane] = exb;
            __syncwarp();
            if (lane < nt) {
                const int t = t0 + lane;
                const int slot = lane < ng ? 0 : 1, grp = lane - slot * ng;
                double v = 0.0;
                float ex = 0.f;
                for (int m = 0; PART != LEAF_FAR && m < sp; m++) {
                    v += red[wib][slot][grp + m * ng];
                    ex += redf[wib][slot][grp + m * ng];
                }
                if (lap && PART != LEAF_FAR) {
                    // the skipped charges leave log2(w^2) * sum(tau); the one skipped
                    // pair is almost always the target itself: take its FP64 charge
                    const double tau_t = A.taus[t];
                    const double exd = ex == (float)tau_t ? tau_t : (double)ex;
                    v += lw * (tsum - exd);
                }
                const double pxd = A.xs[t] - cx, pyd = A.ys[t] - cy;
                // far field (L2P) in FP64
                double far = 0.0;
                if (l >= 2 && PART != LEAF_NEAR) {
                    const double zx = pxd * sc, zy = pyd * sc;
                    if (taylor && zx * zx + zy * zy <= 0.5625) {
                        // Horner: orders P..9 in FP32 (weighted by |z/rho|^9 < 0.008 where
                        // used), then 8..1 in FP64
                        const float zxf = (float)zx, zyf = (float)zy;
                        float fr = qf[R - 2], fi = qf[R - 1];
                        for (int jj = KIFMM_TAYLOR_P - 1; jj >= 9; jj--) {
                            const float nr = fmaf(fr, zxf, fmaf(-fi, zyf, qf[2 * jj - 1]));
                            const float ni = fmaf(fr, zyf, fmaf(fi, zxf, qf[2 * jj]));
                            fr = nr;
                            fi = ni;
                        }
                        double sr = fr, si = fi;
                        for (int jj = 8; jj >= 1; jj--) {
                            double nr = fma(sr, zx, fma(-si, zy, qd[2 * jj - 1]));
                            double ni = fma(sr, zy, fma(si, zx, qd[2 * jj]));
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
                if (PART == LEAF_BOTH) A.pots[t] = v * (double)gsum_scale<KIND>() + far;
                else if (PART == LEAF_NEAR) A.pots[t] = v * (double)gsum_scale<KIND>();
                else A.pots[t] += far;
            }
            __syncwarp();
        }
    }
}

// One warp per leaf.  With `split` (a leaf list smaller than one wave of the
// GPU, where the kernel lasts as long as its heaviest leaf) warps nlist ..
// nlist + *nsplit - 1 take the tiles after the first of the leaves in
// split_list, so a leaf of more than 32 points runs on two warps.
template <int KIND, bool SPLIT, int PART = LEAF_BOTH>
__global__ void __launch_bounds__(32 * LEAF_WARPS, LEAF_BLOCKS_PER_SM)
    k_leaf_eval_f(PassArgs A, int64_t nlist, const int32_t *__restrict__ split_list,
                  const unsigned *__restrict__ nsplit) {
    pdl_trigger();
    pdl_wait();
    const int64_t wstride = (int64_t)gridDim.x * LEAF_WARPS;
    if (!SPLIT) {
        for (int64_t w = (int64_t)blockIdx.x * LEAF_WARPS + (threadIdx.x >> 5); w < nlist; w += wstride)
            leaf_eval_f_leaf<KIND, PART>(A, w);
        return;
    }
    const int64_t total = nlist + *nsplit;
    for (int64_t w = (int64_t)blockIdx.x * LEAF_WARPS + (threadIdx.x >> 5); w < total; w += wstride) {
        const bool first = w < nlist;
        leaf_eval_f_leaf<KIND>(A, first ? w : (int64_t)split_list[w - nlist], first ? 0 : 1, first ? 1 : 1 << 20);
    }
}

// The far field of the Laplace leaves after a near-only pass (LEAF_NEAR), with
// every lane busy: one block per 32 consecutive leaves of one level (the
// k_leaf_taylor tiling), each thread a target of those leaves.  The leaves'
// Taylor coefficients (written by k_leaf_taylor) are staged in shared memory,
// orders >= 9 as FP32 and orders <= 8 as FP64, and the Horner L2P is the
// one of leaf_eval_f_leaf step for step, so the sum added to the near field
// in pots is the same; targets beyond the series radius take the direct sum
// over the equivalent points.  Replaces the far-only warp-per-leaf pass,
// whose Horner ran on about half the lanes.
constexpr int FT_THREADS = 128;
__global__ void __launch_bounds__(FT_THREADS) k_leaf_far_taylor(TaylorArgs T) {
    constexpr int R = 2 * KIFMM_TAYLOR_P + 1;
    __shared__ float qf[32][R + 1];
    __shared__ double qd[32][17];  // orders 0..8
    __shared__ double scx[32], scy[32], ssc[32];
    __shared__ int sbot[32], spre[33], snode[32], slev[32];
    const PassArgs &A = T.A;
    pdl_trigger();
    const int64_t b = blockIdx.x;
    int l = T.lmin;
    while (l < T.lmax && T.toff[l + 1] <= b) l++;
    const int64_t w0 = T.loff[l] + (b - T.toff[l]) * 32;
    const int nt = (int)min((int64_t)32, T.loff[l + 1] - w0);
    const int tid = threadIdx.x;
    pdl_wait();  // coefficients from k_leaf_taylor; near field in pots
    if (tid < 32) {
        int cnt = 0;
        if (tid < nt) {
            const int32_t *rec = A.leaf_rec + (w0 + tid) * LEAF_REC_WORDS;
            const int lv = rec[LR_LEVEL];
            const uint64_t key = (uint64_t)(uint32_t)rec[LR_KEY_LO] | ((uint64_t)(uint32_t)rec[LR_KEY_HI] << 32);
            const double wl = ldexp(A.W, -lv);
            scx[tid] = A.root + ((double)compact2(key >> 1) + 0.5) * wl;
            scy[tid] = A.root + ((double)compact2(key) + 0.5) * wl;
            ssc[tid] = 1.0 / wl;
            sbot[tid] = rec[LR_BOT];
            snode[tid] = rec[LR_NODE];
            slev[tid] = lv;
            cnt = rec[LR_TOP] - rec[LR_BOT];
        }
        int v = cnt;  // inclusive scan of the leaves' point counts
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (tid >= o) v += u;
        }
        spre[tid + 1] = v;
        if (tid == 0) spre[0] = 0;
    }
    for (int i = tid; i < nt * R; i += FT_THREADS) {
        const int n = i / R, r = i - n * R;
        const double c = T.coef[(w0 + n) * R + r];
        qf[n][r] = (float)c;
        if (r < 17) qd[n][r] = c;
    }
    __syncthreads();
    const int total = spre[nt];
    for (int i = tid; i < total; i += FT_THREADS) {
        int n = 0;  // the leaf of flat target i: the last n with spre[n] <= i
        for (int step = 16; step; step >>= 1)
            if (n + step < nt && spre[n + step] <= i) n += step;
        const int t = sbot[n] + (i - spre[n]);
        const double pxd = A.xs[t] - scx[n], pyd = A.ys[t] - scy[n];
        const double zx = pxd * ssc[n], zy = pyd * ssc[n];
        double far;
        if (zx * zx + zy * zy <= 0.5625) {
            const float zxf = (float)zx, zyf = (float)zy;
            float fr = qf[n][R - 2], fi = qf[n][R - 1];
            for (int jj = KIFMM_TAYLOR_P - 1; jj >= 9; jj--) {
                const float nr = fmaf(fr, zxf, fmaf(-fi, zyf, qf[n][2 * jj - 1]));
                const float ni = fmaf(fr, zyf, fmaf(fi, zxf, qf[n][2 * jj]));
                fr = nr;
                fi = ni;
            }
            double sr = fr, si = fi;
            for (int jj = 8; jj >= 1; jj--) {
                double nr = fma(sr, zx, fma(-si, zy, qd[n][2 * jj - 1]));
                double ni = fma(sr, zy, fma(si, zx, qd[n][2 * jj]));
                sr = nr;
                si = ni;
            }
            far = qd[n][0] + (sr * zx - si * zy);
        } else {
            // direct FP64 sum over the equivalent points (targets outside the series radius)
            const int lv = slev[n], g = snode[n];
            const double *lgd = A.ops + (size_t)lv * A.stride + A.off_large;
            const double *inv = A.ops + (size_t)lv * A.stride + A.off_inv;
            const double *u = A.udown + (size_t)g * A.Q;
            far = 0.0;
            for (int q = 0; q < A.Q; q++) {
                double qq = 0.0;
                for (int c = 0; c < A.Q; c++) qq = fma(inv[q * A.Q + c], u[c], qq);
                double dx = pxd - lgd[q], dy = pyd - lgd[A.Q + q];
                far = fma(green_d(A.kind, A.k, dx * dx + dy * dy), qq, far);
            }
        }
        A.pots[t] += far;
    }
}

// the leaves of more than 32 points (their tiles after the first), for the
// split form of k_leaf_eval_f
__global__ void k_leaf_split_list(const int32_t *__restrict__ rec, int64_t nlist, int32_t *__restrict__ out,
                                  unsigned *__restrict__ count) {
    const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool big = w < nlist && rec[w * LEAF_REC_WORDS + LR_TOP] - rec[w * LEAF_REC_WORDS + LR_BOT] > 32;
    const unsigned peers = __ballot_sync(0xffffffffu, big);
    unsigned base = 0;
    if ((threadIdx.x & 31) == 0 && peers) base = atomicAdd(count, (unsigned)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (big) out[base + __popc(peers & ((1u << (threadIdx.x & 31)) - 1))] = (int32_t)w;
}

// The leaf pass of several plans in one launch (serving batches): warp w of
// the grid takes leaf w - off[r] of plan r, off[r] <= w < off[r + 1].
template <int KIND>
__global__ void __launch_bounds__(32 * LEAF_WARPS, LEAF_BLOCKS_PER_SM)
    k_leaf_eval_f_batch(const PassArgs *__restrict__ args, const int64_t *__restrict__ off, int nplan) {
    pdl_trigger();
    pdl_wait();
    const int64_t w = (int64_t)blockIdx.x * LEAF_WARPS + (threadIdx.x >> 5);
    int lo = 0, hi = nplan;  // the last r with off[r] <= w
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= w) lo = mid;
        else hi = mid;
    }
    if (w < off[nplan]) leaf_eval_f_leaf<KIND>(args[lo], w - off[lo]);
}

// Separate targets (class_fmm.py:379-399 with targets other than the
// sources), one thread per target in Morton order (sort_targets): descent to
// the target's leaf, L2P from the leaf's equivalent density (k_leaf_den, in
// FP64), P2P over the leaf's colleagues in FP32 (pairs at distance 0 skipped),
// result written to the target's own position.  Neighbouring lanes mostly
// share a leaf, so node tables and near sources are read once per warp.
__global__ void k_leaf_den(PassArgs A, int64_t nn, double *__restrict__ den) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5, ws = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int Q = A.Q;
    for (int64_t g = w0; g < nn; g += ws) {
        const int l = A.nlev[g];
        if ((A.nflag[g] & NF_SPLIT) || l < 2) continue;
        const double *inv = A.ops + (size_t)l * A.stride + A.off_inv;
        const double *u = A.udown + (size_t)g * Q;
        for (int q = lane; q < Q; q += 32) {
            double s = 0.0;
            for (int c = 0; c < Q; c++) s = fma(inv[q * Q + c], u[c], s);
            den[(size_t)g * Q + q] = s;
        }
    }
}

template <int KIND>
__global__ void k_eval_targets_s(PassArgs A, const double *__restrict__ tx, const double *__restrict__ ty,
                                 const int32_t *__restrict__ order, int64_t n, const double *__restrict__ den,
                                 double *__restrict__ pot) {
    const float kk = (float)A.k;
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
        const float rx = (float)(px - cx), ry = (float)(py - cy);
        double far = 0.0;  // L2P in FP64
        if (l >= 2) {
            const double *lgd = A.ops + (size_t)l * A.stride + A.off_large;
            const double *dg = den + (size_t)g * A.Q;
            for (int q = 0; q < A.Q; q++) {
                const double dx = (px - cx) - lgd[q], dy = (py - cy) - lgd[A.Q + q];
                far = fma(green_d(A.kind, A.k, dx * dx + dy * dy), dg[q], far);
            }
        }
        float acc = 0.f;
        for (int d = 0; d < 9; d++) {
            const int c = A.ncoll[9 * (size_t)g + d];
            if (c < 0) continue;
            for (int s = A.nbot[c]; s < A.ntop[c]; s++) {
                const float dx = rx - (float)(A.xs[s] - cx), dy = ry - (float)(A.ys[s] - cy);
                const float r2 = fmaf(dx, dx, dy * dy);
                if (r2 > 0.f) acc = fmaf((float)A.taus[s], gsum_term<KIND>(r2, kk), acc);
            }
        }
        pot[order[i]] = (double)(acc * gsum_scale<KIND>()) + far;
    }
}

void sort_targets(kifmm_plan *P, const double *tx, const double *ty, int64_t n);  // tree.cu

void launch_leaf_den(kifmm_plan *P, const PassArgs &A) {
    const int64_t nn = P->n_nodes;
    P->node_den.alloc((size_t)nn * P->Q);
    k_leaf_den<<<grid_for(nn * 32, 256, P->num_sms * 16), 256, 0, P->stream>>>(A, nn, P->node_den.p);
    KIFMM_LAUNCHED();
}

// m2l_tc.cu / passes.cu
void run_m2l_tensor(kifmm_plan *P, const PassArgs &A);
void launch_p2m_d(kifmm_plan *P, const PassArgs &A);
void launch_leaf_eval_d(kifmm_plan *P, const PassArgs &A, int check_self);
void launch_eval_targets_d(kifmm_plan *P, const PassArgs &A, const double *tx, const double *ty, int64_t n,
                           int check_self, double *pot);
void launch_m2m_d(kifmm_plan *P, const PassArgs &A, int l);
void launch_l2l_d(kifmm_plan *P, const PassArgs &A, int l);
void run_m2m_levels(kifmm_plan *P, const PassArgs &A);
void run_l2l_levels(kifmm_plan *P, const PassArgs &A);

// P2M and M2M of the mixed apply
void near_launch(kifmm_plan *P);
void mixed_upward(kifmm_plan *P, const PassArgs &A) {
    if (P->n_p2m_list) {
        PhaseScope ph(P, KIFMM_PHASE_P2M);
        if (planned_ready(P)) launch_planned_p2m(P, A);
        else launch_p2m_d(P, A);
    }
    ops_wait_now(P);  // the P2M reads only the check circles
    PhaseScope ph(P, KIFMM_PHASE_M2M);
    run_m2m_levels(P, A);
}

// the L2L chain after the M2L
void mixed_l2l(kifmm_plan *P, const PassArgs &A) {
    PhaseScope ph(P, KIFMM_PHASE_L2L);
    run_l2l_levels(P, A);
}

void run_passes_mixed(kifmm_plan *P) {
    const int Q = P->Q, L = P->L;
    if (L < 3) return;  // expansions cleared by run_upward_downward
    // the near field at the sources on a low-priority stream, the far-field
    // chain below on a high-priority one (launches and allocations swapped
    // there, joined back into the plan's stream at the end)
    const bool near = near_possible(P);
    HighPriorityFork fork(P, near);
    PassArgs A = make_pass_args(P);
    mixed_upward(P, A);
    if (near) near_launch(P);  // after the M2M chain, under the M2L and L2L
    if (P->opt.m2l == KIFMM_M2L_FP32) {
        PhaseScope ph(P, KIFMM_PHASE_M2L);
        const int thr = ((4 * Q + 31) / 32) * 32;
        const size_t smem = (size_t)M2LF_TE * 4 * Q * sizeof(float);
        ensure_dyn_smem(k_m2l_f, smem);
        for (int l = 1; l <= L - 2; l++) {
            int64_t ne = P->lt.ne[l];
            if (!ne) continue;
            k_m2l_f<<<(unsigned)((ne + M2LF_TE - 1) / M2LF_TE), thr, smem, P->stream>>>(A, l);  // (the far stream)
            KIFMM_LAUNCHED();
        }
        return;
    }
    {
        PhaseScope ph(P, KIFMM_PHASE_M2L);
        run_m2l_tensor(P, A);  // all levels at once
    }
    mixed_l2l(P, A);
}

// The arguments of the FP32 leaf kernel; for the Laplace kernel this first
// launches the Taylor coefficients of the leaves' local expansions.
// the 32-leaf tiles of the leaves at levels >= 2 (k_leaf_taylor, k_leaf_far_taylor)
static TaylorArgs taylor_tiling(kifmm_plan *P, const PassArgs &A, int64_t *ntiles) {
    TaylorArgs T{};
    T.A = A;
    T.list = P->leaf_list.p;
    T.coef = P->leaf_coef.p;
    T.lmin = 2;
    T.lmax = P->L - 1;
    int64_t tiles = 0;
    for (int l = 0; l <= MAX_LEVELS; l++) {
        T.loff[l] = P->leaf_loff[l];
        T.toff[l] = tiles;
        if (l >= T.lmin && l <= T.lmax && l < MAX_LEVELS) tiles += (P->leaf_loff[l + 1] - P->leaf_loff[l] + 31) / 32;
    }
    *ntiles = tiles;
    return T;
}

PassArgs mixed_leaf_args(kifmm_plan *P) {
    PassArgs A = make_pass_args(P);
    if (P->kern.kind == KIFMM_KERNEL_LAPLACE && P->l2p_taylor.p && P->L >= 3) {
        constexpr int R = 2 * KIFMM_TAYLOR_P + 1;
        KIFMM_REQUIRE(P->Q % 4 == 0, KIFMM_ERR_ARG, "mixed Laplace form: Nequiv must be a multiple of 4");
        P->leaf_coef.alloc((size_t)P->n_leaf_list * R);
        A.leaf_coef = P->leaf_coef.p;
        int64_t tiles = 0;
        TaylorArgs T = taylor_tiling(P, A, &tiles);
        if (tiles) {
            const size_t smem = ((size_t)P->Q * pad4mod16(8 * TY_MTR) + 32 * (size_t)pad4mod16(P->Q) + 32 * (size_t)R) *
                                sizeof(double);
            ensure_dyn_smem(k_leaf_taylor, smem);
            launch_pdl(k_leaf_taylor, dim3((unsigned)tiles), dim3(TY_THREADS), smem, P->stream, T);
        }
    }
    return A;
}

void run_eval_sources_mixed(kifmm_plan *P, int check_self) {
    if (!P->n_leaf_list) return;
    PhaseScope ph(P, KIFMM_PHASE_LEAF);
    if (P->opt.near_fp64) {
        launch_leaf_eval_d(P, make_pass_args(P), check_self);
        return;
    }  // FP32 form: coincident pairs always contribute zero
    PassArgs A = mixed_leaf_args(P);
    if (P->near_pending) {  // the near field is in P->pots (near_launch): add the far field
        KIFMM_CUDA(cudaStreamWaitEvent(P->stream, P->near_done, 0));
        P->near_pending = false;
        if (A.leaf_coef) {  // Laplace: every leaf of level >= 2 has its Taylor coefficients
            int64_t tiles = 0;
            TaylorArgs T = taylor_tiling(P, A, &tiles);
            if (tiles) launch_pdl(k_leaf_far_taylor, dim3((unsigned)tiles), dim3(FT_THREADS), 0, P->stream, T);
            return;
        }
        const dim3 grid((unsigned)((P->n_leaf_list + LEAF_WARPS - 1) / LEAF_WARPS)), block(32 * LEAF_WARPS);
        if (P->kern.kind == KIFMM_KERNEL_LAPLACE)
            launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_LAPLACE, false, LEAF_FAR>, grid, block, 0, P->stream, A,
                       P->n_leaf_list, (const int32_t *)nullptr, (const unsigned *)nullptr);
        else
            launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_MOD_HELMHOLTZ, false, LEAF_FAR>, grid, block, 0, P->stream, A,
                       P->n_leaf_list, (const int32_t *)nullptr, (const unsigned *)nullptr);
        return;
    }
    // fewer leaves than one wave of warps: split the big ones over two warps
    const int64_t nl = P->n_leaf_list;
    const bool split = nl < (int64_t)P->num_sms * LEAF_BLOCKS_PER_SM * LEAF_WARPS / 2;
    const int32_t *slist = nullptr;
    const unsigned *scount = nullptr;
    if (split) {
        P->leaf_split.alloc((size_t)nl);
        unsigned *cnt = (unsigned *)(P->scal.p + KIFMM_SCAL_LEAF_SPLIT);
        KIFMM_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), P->stream));
        k_leaf_split_list<<<(unsigned)((nl + 255) / 256), 256, 0, P->stream>>>(P->leaf_rec.p, nl, P->leaf_split.p,
                                                                                cnt);
        KIFMM_LAUNCHED();
        slist = P->leaf_split.p;
        scount = cnt;
    }
    const int64_t warps = split ? 2 * nl : nl;
    unsigned gr = (unsigned)std::min<int64_t>((warps + LEAF_WARPS - 1) / LEAF_WARPS, 1ll << 30);
    const dim3 grid(gr), block(32 * LEAF_WARPS);
    if (P->kern.kind == KIFMM_KERNEL_LAPLACE) {
        if (split) launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_LAPLACE, true>, grid, block, 0, P->stream, A, nl, slist, scount);
        else launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_LAPLACE, false>, grid, block, 0, P->stream, A, nl, slist, scount);
    } else {
        if (split)
            launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_MOD_HELMHOLTZ, true>, grid, block, 0, P->stream, A, nl, slist, scount);
        else
            launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_MOD_HELMHOLTZ, false>, grid, block, 0, P->stream, A, nl, slist,
                       scount);
    }
}

// The near field at the sources (P2P of every leaf over its colleagues) needs
// only the sorted points and charges, none of the expansions, so the apply
// runs it on a stream of its own while the far-field chain leaves SMs idle,
// and the evaluation at the sources adds only the far field (LEAF_FAR).
// Mixed FP32 near field, where the near sum does not depend on check_self
// (coincident pairs contribute zero); not inside a stream capture and not for
// leaf lists smaller than one wave (those split big leaves over two warps
// instead).  A later evaluation at other targets leaves the pass unused.
// The near pass runs on a stream of the lowest priority and the far-field
// chain on one of the highest, and the pass starts after the M2M chain, under
// the source slicing, M2L and L2L: started with the apply its blocks, filling
// every SM, held off the M2M chain's small level launches even with the
// priorities (M2M 0.086 -> 0.18 ms at 1M points).  Measured per step against
// the single leaf pass after the chain: 1M mixture 1.005 -> 0.953 ms (0.971-
// 0.994 when started with the apply), 4M uniform 2.446 -> 2.444 ms, 2M K0
// annulus 6.02 -> 5.20 ms (the K0 near field is several times longer than the
// chain, which runs under it).

// the plan's near stream (lowest priority) and far stream (highest), once,
// from the per-device pool
void aux_streams_acquire(int device, cudaStream_t *near, cudaStream_t *far);  // capi.cu: per-device pool
void ensure_aux_streams(kifmm_plan *P) {
    if (P->near_stream) return;
    aux_streams_acquire(P->device, &P->near_stream, &P->far_stream);
    for (cudaEvent_t *e : {&P->near_fork, &P->near_done, &P->far_fork, &P->far_done})
        KIFMM_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
}

bool near_possible(kifmm_plan *P) {
    const int64_t nl = P->n_leaf_list;
    if (P->opt.precision != KIFMM_PREC_MIXED || P->opt.near_fp64 || P->opt.planned || P->cplx || nl <= 0)
        return false;
    if (P->kern.kind != KIFMM_KERNEL_LAPLACE && P->kern.kind != KIFMM_KERNEL_MOD_HELMHOLTZ) return false;
    if (nl < (int64_t)P->num_sms * LEAF_BLOCKS_PER_SM * LEAF_WARPS / 2) return false;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    KIFMM_CUDA(cudaStreamIsCapturing(P->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) return false;
    ensure_aux_streams(P);
    return true;
}

// the near pass, forked from the plan's stream at this point
void near_launch(kifmm_plan *P) {
    const int64_t nl = P->n_leaf_list;
    KIFMM_CUDA(cudaEventRecord(P->near_fork, P->stream));
    KIFMM_CUDA(cudaStreamWaitEvent(P->near_stream, P->near_fork, 0));
    PassArgs A = make_pass_args(P);
    const dim3 grid((unsigned)((nl + LEAF_WARPS - 1) / LEAF_WARPS)), block(32 * LEAF_WARPS);
    {
        struct Swap {  // the phase timer's events go to the near stream
            kifmm_plan *P;
            cudaStream_t main;
            Swap(kifmm_plan *p) : P(p), main(p->stream) { P->stream = P->near_stream; }
            ~Swap() { P->stream = main; }
        } sw(P);
        PhaseScope ph(P, KIFMM_PHASE_LEAF);
        if (P->kern.kind == KIFMM_KERNEL_LAPLACE)
            launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_LAPLACE, false, LEAF_NEAR>, grid, block, 0, P->near_stream, A, nl,
                       (const int32_t *)nullptr, (const unsigned *)nullptr);
        else
            launch_pdl(k_leaf_eval_f<KIFMM_KERNEL_MOD_HELMHOLTZ, false, LEAF_NEAR>, grid, block, 0, P->near_stream, A,
                       nl, (const int32_t *)nullptr, (const unsigned *)nullptr);
    }
    KIFMM_CUDA(cudaEventRecord(P->near_done, P->near_stream));
    P->near_pending = true;
}

// a near-field pass in flight is waited for and dropped (a new tree or apply
// replaces the buffers it reads and writes)
void near_join(kifmm_plan *P) {
    if (!P->near_pending) return;
    KIFMM_CUDA(cudaStreamWaitEvent(P->stream, P->near_done, 0));
    P->near_pending = false;
}

// the FP32 leaf pass of several plans of one kernel kind in one launch
void launch_leaf_f_batch(int kind, const PassArgs *dargs, const int64_t *doff, int nplan, int64_t nleaf,
                         cudaStream_t s) {
    const int64_t blocks = (nleaf + LEAF_WARPS - 1) / LEAF_WARPS;
    KIFMM_REQUIRE(blocks > 0 && blocks < (1ll << 31), KIFMM_ERR_ARG, "batch leaf pass: bad leaf count");
    if (kind == KIFMM_KERNEL_LAPLACE)
        k_leaf_eval_f_batch<KIFMM_KERNEL_LAPLACE><<<(unsigned)blocks, 32 * LEAF_WARPS, 0, s>>>(dargs, doff, nplan);
    else
        k_leaf_eval_f_batch<KIFMM_KERNEL_MOD_HELMHOLTZ><<<(unsigned)blocks, 32 * LEAF_WARPS, 0, s>>>(dargs, doff,
                                                                                                      nplan);
    KIFMM_LAUNCHED();
}

void run_eval_targets_mixed(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self,
                            double *pot) {
    PassArgs A = make_pass_args(P);
    if (P->opt.near_fp64) {
        launch_eval_targets_d(P, A, tx, ty, n, check_self, pot);
        return;
    }
    sort_targets(P, tx, ty, n);
    launch_leaf_den(P, A);
    const unsigned gr = grid_for(n, 128, P->num_sms * 16);
    if (P->kern.kind == KIFMM_KERNEL_LAPLACE)
        k_eval_targets_s<KIFMM_KERNEL_LAPLACE><<<gr, 128, 0, P->stream>>>(A, P->txs.p, P->tys.p, P->tperm.p, n,
                                                                          P->node_den.p, pot);
    else
        k_eval_targets_s<KIFMM_KERNEL_MOD_HELMHOLTZ><<<gr, 128, 0, P->stream>>>(A, P->txs.p, P->tys.p, P->tperm.p,
                                                                                n, P->node_den.p, pot);
    KIFMM_LAUNCHED();
}

}  // namespace kifmm
