// m2l_tc.cu -- M2L on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// Reference: the M2L of FMM.build_expansions, class_fmm.py:336-343 -- eight
// dense GEMMs CM2LS[d] @ RSEQD.T per level, then a scatter into the target
// sibling groups.  Here the GEMM is target-centric and gathers its operand:
//
//   u_down(children of p) = sum_{d != centre} C_d . u_up(children of p + d)
//
// with C_d = CM2LS_d . blockdiag(Inv) (4Q x 4Q, FP64, operators.cu).  As a
// GEMM: D[rows, targets] = A[rows, 8 x 4Q] . B[targets, 8 x 4Q]^T where B's
// columns are gathered per target from its eight neighbour groups.  A CTA
// owns TN target groups (96 for int8: five accumulators of 96 columns fill
// the 512 TMEM columns of an SM) and one 128-row M tile.  Its work is a list
// of stages (direction with a source in the tile, 64-byte K chunk) that runs
// through a ring of TC_STAGES shared-memory slots, warp-specialised:
//   * warps 0 .. TC_GWARPS-1 gather the sources' pre-sliced K chunks into a slot (16-byte
//     cp.async copies) and arrive on its B-full barrier once they landed;
//   * one thread of warp 4 copies the operator chunk into the slot with one
//     bulk copy (A-full barrier, transaction bytes), waits for both, issues the
//     stage's MMA chain and commits it to the slot's empty barrier, which
//     frees the slot for the gather warps and for its own next operator copy;
//   * after the last stage, the gather warps read TMEM (warp w its 32 lanes
//     of quarter w % 4, a share of the columns) and write the FP64 results.
// Operands sit in the UMMA K-major, no-swizzle core-matrix layout.
//
// Forms:
//   INT8 (default): A row-scaled and B column-scaled by powers of two into
//     (-1, 1), each split into five signed 7-bit slices (x = sum_i s_i 2^-7(i+1)).
//     kind::i8 products accumulate EXACTLY in int32; the 15 slice products
//     with i + j <= 4 go to five TMEM accumulators (one per power of two) and
//     are recombined in FP64.  Error ~2^-35 of the row/column scales: the
//     FP64 result, without the FP32-accumulation floor that the
//     measured ~10x cancellation in these sums puts near 1e-6.
//   BF16X3 / FP16X3: hi/lo splits, three kind::f16 products (hi.hi, hi.lo,
//     lo.hi) accumulated in FP32 in TMEM (the fp16 operator pre-scaled by 2^12).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "passes.cuh"
#include "async_copy.cuh"

namespace kifmm {

enum TcForm { TC_INT8 = 0, TC_BF16 = 1, TC_FP16 = 2, TC_I8S4 = 3 };
// NS slices per operand, EB bytes per element, KSTEP elements per MMA, NACC
// accumulators, TN target groups per CTA (MMA N), NCOLS TMEM columns allocated
template <int F> struct TcTraits;
template <> struct TcTraits<TC_INT8> { static constexpr int NS = 5, EB = 1, KSTEP = 32, NACC = 5, TN = 96, NCOLS = 512; };
template <> struct TcTraits<TC_BF16> { static constexpr int NS = 2, EB = 2, KSTEP = 16, NACC = 1, TN = 64, NCOLS = 64; };
template <> struct TcTraits<TC_FP16> { static constexpr int NS = 2, EB = 2, KSTEP = 16, NACC = 1, TN = 64, NCOLS = 64; };
template <> struct TcTraits<TC_I8S4> { static constexpr int NS = 4, EB = 1, KSTEP = 32, NACC = 4, TN = 128, NCOLS = 512; };
// the integer (kind::i8) forms
template <int F> __host__ __device__ constexpr bool tc_int() { return F == TC_INT8 || F == TC_I8S4; }

constexpr int TC_M = 128;        // MMA M: operator rows per tile (TMEM lanes)
#ifndef KIFMM_TC_KCB
#define KIFMM_TC_KCB 64
#endif
#ifndef KIFMM_TC_STAGES
#define KIFMM_TC_STAGES 3
#endif
constexpr int TC_KCB = KIFMM_TC_KCB;        // bytes of K per slice row and stage (64: 2 MMA K steps)
constexpr int TC_STAGES = KIFMM_TC_STAGES;  // shared-memory ring slots
#ifndef KIFMM_TC_GWARPS
#define KIFMM_TC_GWARPS 8
#endif
// gather / epilogue warps: warp w reads TMEM lanes 32 (w % 4) .. + 31 and every
// (TC_GWARPS / 4)-th 16-column group of the accumulators from group w / 4
constexpr int TC_GWARPS = KIFMM_TC_GWARPS;
static_assert(TC_GWARPS % 4 == 0, "epilogue warps cover the four TMEM lane quarters equally");
constexpr int TC_THREADS = 32 * (TC_GWARPS + 1);
template <int F>
constexpr bool tc_traits_ok() {
    using TR = TcTraits<F>;
    return TR::TN % 16 == 0 && TR::TN >= 16 && TR::TN <= 256 && TR::NACC * TR::TN <= TR::NCOLS &&
           TR::TN <= 32 * TC_GWARPS && TR::TN % 32 == 0 && (TC_KCB / TR::EB) % TR::KSTEP == 0;
}
static_assert(tc_traits_ok<TC_INT8>() && tc_traits_ok<TC_BF16>() && tc_traits_ok<TC_FP16>() &&
                  tc_traits_ok<TC_I8S4>(), "tile shapes");
constexpr double FP16_PRESCALE = 4096.0;

struct TcGeom {
    int Q4, MP, MT, KP, NKC;   // rows, padded rows, M tiles, padded K per direction, K chunks
    size_t slice_bytes;        // one slice of one A tile chunk: 128 x TC_KCB bytes
    size_t level_bytes;        // all A slices of one level
};

template <int F>
static TcGeom tc_geom(int Q) {
    constexpr int KCE = TC_KCB / TcTraits<F>::EB;
    TcGeom g;
    g.Q4 = 4 * Q;
    g.MP = (g.Q4 + TC_M - 1) / TC_M * TC_M;
    g.MT = g.MP / TC_M;
    g.KP = (g.Q4 + KCE - 1) / KCE * KCE;
    g.NKC = g.KP / KCE;
    g.slice_bytes = (size_t)TC_M * TC_KCB;
    g.level_bytes = (size_t)9 * g.MT * g.NKC * TcTraits<F>::NS * g.slice_bytes;
    return g;
}

// byte offset of element (row, k) in a core-matrix tile of `rows` rows:
// 16-byte K chunks, 8-row groups, chunk-major (K-major, no swizzle).
__host__ __device__ __forceinline__ uint32_t core_off(int row, int k, int rows, int eb) {
    int kb = k * eb;
    return (uint32_t)(((kb >> 4) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (kb & 15));
}

// ------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}
template <int F>
__device__ __forceinline__ uint32_t instr_desc() {
    // c_format [4,6), a_format [7,10), b_format [10,13), N>>3 [17,23), M>>4 [24,29)
    uint32_t fmt = tc_int<F>() ? ((2u << 4) | (1u << 7) | (1u << 10))    // s32 <- s8 x s8
                 : F == TC_BF16 ? ((1u << 4) | (1u << 7) | (1u << 10))    // f32 <- bf16 x bf16
                                : (1u << 4);                              // f32 <- f16 x f16
    return fmt | ((uint32_t)(TcTraits<F>::TN >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}
template <int F>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    if (tc_int<F>()) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
    }
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// power of two with max_abs * 128/127 <= result (1 for zero)
__host__ __device__ __forceinline__ double pow2_scale(double max_abs) {
    if (!(max_abs > 0.0)) return 1.0;
    int e;
    frexp(max_abs * (128.0 / 127.0), &e);
    return ldexp(1.0, e);
}

// split v in (-1, 1) into the form's slices, writing element (row, k) of each
template <int F>
__device__ __forceinline__ void put_slices(unsigned char *tile, size_t slice_bytes, uint32_t off, double v) {
    if (tc_int<F>()) {
        double r = v;
#pragma unroll
        for (int s = 0; s < TcTraits<F>::NS; s++) {
            r *= 128.0;
            double q = rint(r);
            r -= q;
            ((int8_t *)(tile + s * slice_bytes))[off] = (int8_t)q;
        }
    } else if (F == TC_BF16) {
        __nv_bfloat16 hi = __double2bfloat16(v);
        __nv_bfloat16 lo = __double2bfloat16(v - (double)__bfloat162float(hi));
        *(__nv_bfloat16 *)(tile + off) = hi;
        *(__nv_bfloat16 *)(tile + slice_bytes + off) = lo;
    } else {
        double w = v * FP16_PRESCALE;
        __half hi = __double2half(w);
        __half lo = __double2half(w - (double)__half2float(hi));
        *(__half *)(tile + off) = hi;
        *(__half *)(tile + slice_bytes + off) = lo;
    }
}

// ------------------------------------------------ operator slices (precompute)
struct TcOpsArgs {
    const double *ops;     // FP64 level blocks
    size_t stride, off_m2l;
    int Q, L;
    TcGeom g;
    unsigned char *aslices;  // [L][9][MT][NKC][NS][slice]
    double *rowscale;        // [L][MP]
    const unsigned long long *rowmax;  // [L][Q4] largest |value| per row (operators.cu, k_ops_assemble)
};

template <int F>
__global__ void k_tc_slices(TcOpsArgs T) {
    const int l = blockIdx.x, d = blockIdx.y;
    if (l < 2 || d == 4) return;
    const int Q4 = T.g.Q4;
    const double *C = T.ops + (size_t)l * T.stride + T.off_m2l + (size_t)d * Q4 * Q4;
    unsigned char *base = T.aslices + (size_t)l * T.g.level_bytes;
    const size_t sb = T.g.slice_bytes;
    const int total = T.g.MP * T.g.KP;
    // row scale: the power of two above the row's largest |value| over all
    // directions (1 for padding rows); multiplying by its reciprocal is exact
    auto scale_of = [&](int r) {
        return r < Q4 ? pow2_scale(__longlong_as_double((long long)T.rowmax[(size_t)l * Q4 + r])) : 1.0;
    };
    if (d == 0 && blockIdx.z == 0)
        for (int r = threadIdx.x; r < T.g.MP; r += blockDim.x) T.rowscale[(size_t)l * T.g.MP + r] = scale_of(r);
    for (int e = blockIdx.z * blockDim.x + threadIdx.x; e < total; e += gridDim.z * blockDim.x) {
        int r = e % T.g.MP, k = e / T.g.MP;
        double v = (r < Q4 && k < Q4) ? C[(size_t)k * Q4 + r] * (1.0 / scale_of(r)) : 0.0;
        constexpr int KCE = TC_KCB / TcTraits<F>::EB;
        int mt = r / TC_M, kc = k / KCE;
        unsigned char *tile = base + (((size_t)d * T.g.MT + mt) * T.g.NKC + kc) * TcTraits<F>::NS * sb;
        put_slices<F>(tile, sb, core_off(r % TC_M, k % KCE, TC_M, TcTraits<F>::EB), v);
    }
}

// Source groups are sliced once per apply.  INT8: each group gets its own
// scale 2^(7 k_g) (k_g the smallest integer with max|u| * 128/127 <= 2^(7 k_g))
// and five 7-bit slices of u / 2^(7 k_g); a target column whose largest group
// exponent is k_j then uses the group's slice i - (k_j - k_g) as its slice i,
// so B is staged by byte copies.  Float forms store hi/lo of u itself.
struct TcPre {
    unsigned char *slices;   // [n_ent][NS][KP] elements
    int *gexp;               // [n_ent] (INT8)
    const int *src8;         // [n_ent][8] source entry of a split entry per direction (-1: none)
    int KP;
};

template <int F>
__global__ void k_tc_preslice(PassArgs A, int64_t n_ent, TcPre T) {
    using TR = TcTraits<F>;
    pdl_trigger();
    pdl_wait();
    const int lane = threadIdx.x & 31;
    int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (j >= n_ent) return;
    const int Q4 = 4 * A.Q;
    int l = (int)(A.ent[j] >> ENT_LEVEL_SHIFT);
    int64_t cg = A.T.off[l + 1] + 4 * (j - A.T.eoff[l]);
    const double *u = A.uup + (size_t)cg * A.Q;
    unsigned char *out = T.slices + (size_t)j * TR::NS * T.KP * TR::EB;
    if (tc_int<F>()) {
        double m = 0.0;
        for (int c = lane; c < Q4; c += 32) m = fmax(m, fabs(u[c]));
        for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        int kg = 0;
        if (m > 0.0) {
            int e;
            frexp(m * (128.0 / 127.0), &e);  // m * 128/127 < 2^e
            kg = (e >= 0) ? (e + 6) / 7 : -((-e) / 7);
        }
        // X = rint(u 2^(7 NS - 7 kg)), |X| < 2^(7 NS) 127/128 + 1/2, as NS signed
        // base-128 digits: the NS - 1 low ones balanced in [-64, 63] (taken
        // from the bottom with carries), the top one in [-127, 127]; exact
        // integer work after one rounding
        const double scale = ldexp(1.0, 7 * TR::NS - 7 * kg);
        for (int c = lane; c < T.KP; c += 32) {
            long long X = c < Q4 ? __double2ll_rn(u[c] * scale) : 0ll;
#pragma unroll
            for (int i = TR::NS - 1; i > 0; i--) {
                const long long q = ((X + 64) & 127) - 64;
                ((int8_t *)out)[(size_t)i * T.KP + c] = (int8_t)q;
                X = (X - q) >> 7;
            }
            ((int8_t *)out)[c] = (int8_t)X;
        }
        if (lane == 0) T.gexp[j] = kg;
    } else {
        for (int c = lane; c < T.KP; c += 32) {
            double v = c < Q4 ? u[c] : 0.0;
            if (F == TC_BF16) {
                __nv_bfloat16 hi = __double2bfloat16(v);
                ((__nv_bfloat16 *)out)[c] = hi;
                ((__nv_bfloat16 *)out)[T.KP + c] = __double2bfloat16(v - (double)__bfloat162float(hi));
            } else {
                __half hi = __double2half(v);
                ((__half *)out)[c] = hi;
                ((__half *)out)[T.KP + c] = __double2half(v - (double)__half2float(hi));
            }
        }
    }
}


// ------------------------------------------------------------- the kernel
struct TcArgs {
    PassArgs A;
    TcGeom g;
    const unsigned char *aslices;  // all levels
    const double *rowscale;        // all levels [L][MP]
    TcPre pre;
    int lmin, lmax;                // parent levels with targets
    int64_t tile_off[MAX_LEVELS + 1];
    unsigned long long *err;       // set on a timed-out wait
    long long wait_limit;
};

template <int F>
static constexpr size_t tc_stage_a() { return (size_t)TcTraits<F>::NS * TC_M * TC_KCB; }
template <int F>
static constexpr size_t tc_stage_b() { return (size_t)TcTraits<F>::NS * TcTraits<F>::TN * TC_KCB; }
// shared memory: ring (A then B per slot), then per-target tables, then barriers
template <int F>
static constexpr size_t tc_table_off() { return TC_STAGES * (tc_stage_a<F>() + tc_stage_b<F>()); }
template <int F>
static constexpr size_t tc_smem_bytes() {
    constexpr int TN = TcTraits<F>::TN;
    return tc_table_off<F>() + (size_t)TN * 8 * 4 * 2 + (size_t)TN * 8 * 2 + (size_t)TN * 4 + 16 * 4 +
           (3 * TC_STAGES + 2) * 8 + 16;
}

// warp-uniform bounded wait: true once the phase with this parity has completed
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, long long limit) {
    return __any_sync(0xffffffffu, mbar_wait(bar, parity, limit));
}

// column tile `tile` of the M2L of T's plan, by one CTA
template <int F>
__device__ __forceinline__ void m2l_tc_tile(const TcArgs &T, const int64_t tile) {
    using TR = TcTraits<F>;
    constexpr int TN = TR::TN, NS = TR::NS, EB = TR::EB, S = TC_STAGES;
    constexpr int KSTEPS = TC_KCB / EB / TR::KSTEP;
    constexpr uint32_t A_SLICE = TC_M * TC_KCB, B_SLICE = TN * TC_KCB;
    constexpr uint32_t A_STAGE = NS * A_SLICE, B_STAGE = NS * B_SLICE;
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char *sA = tc_smem;                                  // [S][NS][128 x 64 B]
    unsigned char *sB = sA + S * A_STAGE;                         // [S][NS][TN x 64 B]
    int *sgrp = (int *)(tc_smem + tc_table_off<F>());             // [TN][8] source entry per direction
    int *sshift = sgrp + TN * 8;                                  // [TN][8] slice shift (INT8)
    double *stau = (double *)(sshift + TN * 8);                   // [TN] column scale
    long long *sdst = (long long *)(stau + TN);                   // [TN] first u_down element of the target's children
    int *sact = (int *)(sdst + TN);                               // [TN]
    int *sdir = sact + TN;                                        // [8] directions with a source; [8] count; [9] abort
    uint64_t *bars = (uint64_t *)(((uintptr_t)(sdir + 16) + 7) & ~(uintptr_t)7);
    uint32_t *tslot = (uint32_t *)(bars + 3 * S + 1);
    volatile int *abort_flag = sdir + 9;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const PassArgs &A = T.A;
    const int Q = A.Q, Q4 = T.g.Q4, KP = T.pre.KP, NKC = T.g.NKC;

    // which level / column tile / M tile
    int l = T.lmin;
    while (l < T.lmax && T.tile_off[l + 1] <= tile) l++;
    const int64_t lt = tile - T.tile_off[l];
    const int mt = (int)(lt % T.g.MT);
    const int64_t e0 = (lt / T.g.MT) * TN, ne = A.T.ne[l], eoff = A.T.eoff[l];
    const int lt1 = l + 1;  // target level: its operators
    const unsigned char *alev = T.aslices + (size_t)lt1 * T.g.level_bytes;
    const double *rsl = T.rowscale + (size_t)lt1 * T.g.MP;

    if (warp == TC_GWARPS) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TR::NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) sdir[10] = 0;
    __syncthreads();
    if (tid < TN) {  // the tile's targets in M2L target order; sact = 1 + index in the level, 0: none
        const int64_t e = e0 + tid, ej = e < ne ? (int64_t)A.m2l_perm[eoff + e] : -1;
        const bool act = ej >= 0 && !(A.ent[ej] & 1);
        int kcol = -1000000;
        int gs[8];
#pragma unroll
        for (int dd = 0; dd < 8; dd++) gs[dd] = act ? T.pre.src8[ej * 8 + dd] : -1;
#pragma unroll
        for (int dd = 0; dd < 8; dd++) {
            const int grp = gs[dd];
            if (tc_int<F>() && grp >= 0) kcol = max(kcol, T.pre.gexp[grp]);
            sgrp[tid * 8 + dd] = grp;
        }
        if (kcol == -1000000) kcol = 0;
        for (int dd = 0; dd < 8; dd++) {
            const int grp = sgrp[tid * 8 + dd];
            sshift[tid * 8 + dd] = (tc_int<F>() && grp >= 0) ? kcol - T.pre.gexp[grp] : 0;
        }
        stau[tid] = tc_int<F>() ? ldexp(1.0, 7 * kcol) : 1.0;
        sact[tid] = act ? (int)(ej - eoff) + 1 : 0;
        sdst[tid] = act ? (A.T.off[l + 1] + 4 * (ej - eoff)) * (long long)Q : 0;
    }
    if (tid == 0) {
        for (int i = 0; i < S; i++) {
            mbar_init(smem_u32(&bars[i]), 1);                  // A full: the copy's bytes
            mbar_init(smem_u32(&bars[S + i]), 32 * TC_GWARPS); // B full: each gather thread's copies
            mbar_init(smem_u32(&bars[2 * S + i]), 1);          // empty: the stage's MMA commit
        }
        mbar_init(smem_u32(&bars[3 * S]), 1);                  // accumulators complete
        sdir[9] = 0;
    }
    if (tid < TN) {  // directions with a source somewhere in the tile: OR of the targets' masks
        unsigned m = 0;
        for (int dd = 0; dd < 8; dd++) m |= (sgrp[tid * 8 + dd] >= 0 ? 1u : 0u) << dd;
        for (int o = 16; o; o >>= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
        if (lane == 0 && m) atomicOr(&sdir[10], (int)m);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
        const unsigned m = (unsigned)sdir[10];
        int n = 0;
        for (int dd = 0; dd < 8; dd++)
            if (m >> dd & 1u) sdir[n++] = dd;
        sdir[8] = n;
    }
    __syncthreads();
    const uint32_t tmem = *tslot;
    const int nst = sdir[8] * NKC;
    const uint32_t afull0 = smem_u32(&bars[0]), bfull0 = smem_u32(&bars[S]), empty0 = smem_u32(&bars[2 * S]);
    const uint32_t accbar = smem_u32(&bars[3 * S]);

    if (warp == TC_GWARPS) {
        if (lane == 0) {
            // operator chunk of stage st into slot st % S
            auto issue_a = [&](int st) {
                const int d0 = sdir[st / NKC], d = d0 < 4 ? d0 : d0 + 1, kc = st % NKC, slot = st % S;
                const uint32_t bar = afull0 + 8u * slot;
                mbar_expect_tx(bar, A_STAGE);
                bulk_g2s(smem_u32(sA + slot * A_STAGE), alev + (((size_t)d * T.g.MT + mt) * NKC + kc) * A_STAGE, A_STAGE,
                         bar);
            };
            int issued = 0, consumed = 0;
            for (; issued < S && issued < nst; issued++) issue_a(issued);
            const uint32_t idesc = instr_desc<F>();
            constexpr uint32_t a_lbo = (TC_M / 8) * 128, b_lbo = (TN / 8) * 128;
            // descriptors of the ring's first slot; an operand's descriptor is that
            // plus its byte offset / 16 (the start-address field, no carry: smem < 256 KB)
            const uint64_t adesc0 = umma_desc(smem_u32(sA), a_lbo, 128), bdesc0 = umma_desc(smem_u32(sB), b_lbo, 128);
            bool ok = true;
            for (int st = 0; st < nst; st++) {
                const int slot = st % S;
                const uint32_t ph = (uint32_t)(st / S) & 1u;
                if (!mbar_wait(afull0 + 8u * slot, ph, T.wait_limit) || !mbar_wait(bfull0 + 8u * slot, ph, T.wait_limit)) {
                    ok = false;
                    break;
                }
                consumed++;
                fence_after();
                const uint64_t as = adesc0 + ((uint64_t)(slot * A_STAGE) >> 4), bs = bdesc0 + ((uint64_t)(slot * B_STAGE) >> 4);
                const uint32_t later = st != 0;  // the first stage starts every accumulator
#pragma unroll
                for (int ks = 0; ks < KSTEPS; ks++) {
#pragma unroll
                    for (int i = 0; i < NS; i++) {
                        constexpr int JM = tc_int<F>() ? NS - 1 : 1;
#pragma unroll
                        for (int jj = 0; jj <= JM; jj++) {
                            // int8: the 15 slice pairs with i + j <= 4; f16 forms: hi.hi, hi.lo, lo.hi
                            if (tc_int<F>() ? (i + jj > NS - 1) : (i != 0 && jj != 0)) continue;
                            const int acc = tc_int<F>() ? i + jj : 0;
                            const bool first_mma = ks == 0 && i == 0 && (tc_int<F>() || jj == 0);
                            const uint64_t ad = as + ((uint64_t)(i * A_SLICE + ks * 2 * a_lbo) >> 4);
                            const uint64_t bd = bs + ((uint64_t)(jj * B_SLICE + ks * 2 * b_lbo) >> 4);
                            mma_issue<F>(tmem + acc * TN, ad, bd, idesc, first_mma ? later : 1u);
                        }
                    }
                }
                mma_commit(empty0 + 8u * slot);
                // the operator copy of stage st - 1 + S goes into the slot of stage
                // st - 1 once that stage's MMAs (issued before these) are done
                if (st >= 1 && issued < nst) {
                    const int ps = (st - 1) % S;
                    if (!mbar_wait(empty0 + 8u * ps, (uint32_t)((st - 1) / S) & 1u, T.wait_limit)) {
                        ok = false;
                        break;
                    }
                    issue_a(issued++);
                }
            }
            if (!ok) {
                *abort_flag = 1;
                atomicOr(T.err, 1ull);
            }
            mma_commit(accbar);  // completes once every MMA issued above is done
            // operator copies issued but never waited for land before the block leaves
            for (int st = consumed; st < issued; st++) mbar_wait(afull0 + 8u * (st % S), (uint32_t)(st / S) & 1u, kDrainWaitPolls);
        }
        __syncwarp();
    } else {
        // gather warps: the sources' slices of stage st into slot st % S by
        // 16-byte cp.async copies, one commit group per stage; a thread arrives
        // on a slot's B-full barrier once its copies of that stage have landed,
        // checked one stage later so that two stages' copies are in flight
        // a thread takes (target row j, slice i) pairs and copies the row's CH
        // 16-byte chunks; j = 8 jb + t8 with t8 the fastest index, so the 8
        // lanes of a wavefront fill one 128-byte core matrix (no bank conflicts)
        constexpr int CH = TC_KCB / 16, NP = TN * NS, PER = (NP + 32 * TC_GWARPS - 1) / (32 * TC_GWARPS);
        int gdone = 0;  // stages whose copies this thread issued
        for (int st = 0; st < nst; st++) {
            if (*abort_flag) break;
            const int slot = st % S, dd = sdir[st / NKC], kc = st % NKC;
            if (st >= S && !warp_wait(empty0 + 8u * slot, (uint32_t)(st / S - 1) & 1u, T.wait_limit)) {
                if (lane == 0) {
                    *abort_flag = 1;
                    atomicOr(T.err, 1ull);
                }
                break;
            }
            const uint32_t sBs = smem_u32(sB + slot * B_STAGE);
            // absent sources and slices shifted out are copied as zeros
#pragma unroll
            for (int q = 0; q < PER; q++) {
                const int idx = tid + q * 32 * TC_GWARPS;
                if (idx < NP) {
                    const int t8 = idx & 7, jb = (idx >> 3) % (TN / 8), i = idx / TN, j = 8 * jb + t8;
                    const int grp = sgrp[j * 8 + dd], si = i - sshift[j * 8 + dd];
                    const bool has = grp >= 0 && si >= 0 && si < NS;
                    const unsigned char *src =
                        T.pre.slices + (has ? ((size_t)grp * NS + si) * KP * EB + (size_t)kc * TC_KCB : 0);
                    const uint32_t dst = sBs + i * B_SLICE + jb * 128 + t8 * 16;
#pragma unroll
                    for (int c = 0; c < CH; c++)
                        cp_async16(dst + c * (TN / 8) * 128, src + (has ? c * 16 : 0), has ? 16u : 0u);
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
            if (st >= 1) {  // stage st - 1 has landed: make it visible to the tensor core, arrive
                asm volatile("cp.async.wait_group 1;" ::: "memory");
                fence_proxy_async();
                mbar_arrive(bfull0 + 8u * ((st - 1) % S));
            }
            gdone = st + 1;
        }
        // the last stage issued (also after an abort): every copy lands before going on
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (gdone >= 1) {
            fence_proxy_async();
            mbar_arrive(bfull0 + 8u * ((gdone - 1) % S));
        }
    }
    // every thread: the MMAs are complete (or the block gave up) before TMEM is read or freed
    mbar_wait(accbar, 0, kDrainWaitPolls);
    fence_after();
    if (warp < TC_GWARPS && !*abort_flag) {
        const int quarter = warp & 3, row = quarter * 32 + lane, r = mt * TC_M + row;
        const double sig = rsl[r];
#pragma unroll 1
        for (int cc = warp >> 2; cc < TN / 16; cc += TC_GWARPS / 4) {
            double y[16];
#pragma unroll
            for (int c = 0; c < 16; c++) y[c] = 0.0;
            if (nst > 0) {
                uint32_t v[TR::NACC][16];
#pragma unroll
                for (int s = 0; s < TR::NACC; s++)
                    tmem_ld16_nowait(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(s * TN + cc * 16), v[s]);
                tmem_wait_ld();
                if (tc_int<F>()) {
                    // accumulator s carries weight 2^-7(s+2): combine exactly in int64
                    // (|acc| < 2^31, so the sum stays below 2^60), one conversion per column
#pragma unroll
                    for (int c = 0; c < 16; c++) {
                        long long z = 0;
#pragma unroll
                        for (int s = 0; s < TR::NACC; s++) z += (long long)(int32_t)v[s][c] << (7 * (TR::NACC - 1 - s));
                        // exact: z is an integer below 2^60 and the factor a power of two
                        constexpr double kWeight = 1.0 / (double)(1ll << (7 * (TR::NACC + 1)));
                        y[c] = (double)z * kWeight;
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 16; c++)
                        y[c] = (double)__uint_as_float(v[0][c]) * (F == TC_FP16 ? 1.0 / FP16_PRESCALE : 1.0);
                }
            }
            if (r < Q4)
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    const int j = cc * 16 + c;
                    if (sact[j]) A.udown[sdst[j] + r] = y[c] * sig * stau[j];
                }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == TC_GWARPS) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TR::NCOLS));
    }
}

template <int F>
__global__ void __launch_bounds__(TC_THREADS, 1) k_m2l_tc(TcArgs T) {
    pdl_trigger();
    pdl_wait();
    m2l_tc_tile<F>(T, blockIdx.x);
}

// The M2L of several plans in one launch (serving batches): CTA b takes tile
// b - off[r] of plan r, off[r] <= b < off[r + 1].  The plans' arguments are
// read from global memory.
template <int F>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_m2l_tc_batch(const TcArgs *__restrict__ args, const int64_t *__restrict__ off, int nplan) {
    pdl_trigger();
    pdl_wait();
    const int64_t b = blockIdx.x;
    int lo = 0, hi = nplan;  // the last r with off[r] <= b
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= b) lo = mid;
        else hi = mid;
    }
    if (b < off[nplan]) m2l_tc_tile<F>(args[lo], b - off[lo]);
}

// ------------------------------------------------------------ host side
bool uses_tensor_m2l(const kifmm_plan *P) {
    return P->opt.precision == KIFMM_PREC_MIXED &&
           (P->opt.m2l == KIFMM_M2L_INT8 || P->opt.m2l == KIFMM_M2L_INT8X4 || P->opt.m2l == KIFMM_M2L_BF16X3 ||
            P->opt.m2l == KIFMM_M2L_FP16X3);
}

static int form_of(int m2l) {
    return m2l == KIFMM_M2L_BF16X3 ? TC_BF16 : m2l == KIFMM_M2L_FP16X3 ? TC_FP16 : m2l == KIFMM_M2L_INT8X4 ? TC_I8S4 : TC_INT8;
}

template <int F>
static void build_tc_ops_t(kifmm_plan *P) {
    TcGeom g = tc_geom<F>(P->Q);
    P->tc_a.alloc(g.level_bytes * P->L);
    P->tc_rowscale.alloc((size_t)g.MP * P->L);
    TcOpsArgs T{};
    T.ops = P->ops.p;
    T.stride = P->ops_stride;
    T.off_m2l = (size_t)9 * P->Q * P->Q;
    T.Q = P->Q;
    T.L = P->L;
    T.g = g;
    T.aslices = P->tc_a.p;
    T.rowscale = P->tc_rowscale.p;
    T.rowmax = P->tc_rowmax.p;
    k_tc_slices<F><<<dim3(P->L, 9, 8), 256, 0, P->stream>>>(T);
    KIFMM_LAUNCHED();
}

void build_tc_operators(kifmm_plan *P) {
    switch (form_of(P->opt.m2l)) {
        case TC_BF16: build_tc_ops_t<TC_BF16>(P); break;
        case TC_FP16: build_tc_ops_t<TC_FP16>(P); break;
        case TC_I8S4: build_tc_ops_t<TC_I8S4>(P); break;
        default: build_tc_ops_t<TC_INT8>(P); break;
    }
}

// The preslice of P's source expansions (launched on P->stream) and the
// arguments of P's M2L; returns the number of CTA tiles (0: no M2L).
template <int F>
static int64_t tc_prepare_t(kifmm_plan *P, const PassArgs &A, TcArgs &T) {
    using TR = TcTraits<F>;
    TcGeom g = tc_geom<F>(P->Q);
    const int L = P->L;
    if (L < 3 || !P->n_ent) return 0;
    TcPre pre{};
    pre.KP = g.KP;
    P->tc_pre.alloc((size_t)P->n_ent * TR::NS * g.KP * TR::EB);
    P->tc_gexp.alloc(P->n_ent);
    pre.slices = P->tc_pre.p;
    pre.gexp = P->tc_gexp.p;
    pre.src8 = P->m2l_src8.p;  // built with the tree
    launch_pdl(k_tc_preslice<F>, dim3(grid_for(P->n_ent * 32, 256)), dim3(256), 0, P->stream, A, P->n_ent, pre);
    T = TcArgs{};
    T.A = A;
    T.g = g;
    T.aslices = P->tc_a.p;
    T.rowscale = P->tc_rowscale.p;
    T.pre = pre;
    T.err = P->scal.p + KIFMM_SCAL_TC_ERR;
    T.wait_limit = plan_wait_polls(P);
    T.lmin = 1;
    T.lmax = L - 2;
    int64_t tiles = 0;
    for (int l = 0; l <= MAX_LEVELS; l++) {
        T.tile_off[l] = tiles;
        if (l >= T.lmin && l <= T.lmax) tiles += (P->lt.ne[l] + TR::TN - 1) / TR::TN * g.MT;
    }
    return tiles;
}

template <int F>
static void run_m2l_tensor_t(kifmm_plan *P, const PassArgs &A) {
    TcArgs T;
    const int64_t tiles = tc_prepare_t<F>(P, A, T);
    if (!tiles) return;
    size_t smem = tc_smem_bytes<F>();
    ensure_dyn_smem(k_m2l_tc<F>, smem);
    launch_pdl(k_m2l_tc<F>, dim3((unsigned)tiles), dim3(TC_THREADS), smem, P->stream, T);
}

// M2L of every level in one launch (u_down of each split entry's children is
// assigned); the L2L chain runs afterwards.
void run_m2l_tensor(kifmm_plan *P, const PassArgs &A) {
    switch (form_of(P->opt.m2l)) {
        case TC_BF16: run_m2l_tensor_t<TC_BF16>(P, A); break;
        case TC_FP16: run_m2l_tensor_t<TC_FP16>(P, A); break;
        case TC_I8S4: run_m2l_tensor_t<TC_I8S4>(P, A); break;
        default: run_m2l_tensor_t<TC_INT8>(P, A); break;
    }
}

// ---------------------------------------------------- serving batches
int tc_form(const kifmm_plan *P) { return form_of(P->opt.m2l); }
size_t tc_args_bytes() { return sizeof(TcArgs); }

int64_t tc_prepare_batch(kifmm_plan *P, const PassArgs &A, void *args) {
    TcArgs &T = *(TcArgs *)args;
    switch (form_of(P->opt.m2l)) {
        case TC_BF16: return tc_prepare_t<TC_BF16>(P, A, T);
        case TC_FP16: return tc_prepare_t<TC_FP16>(P, A, T);
        case TC_I8S4: return tc_prepare_t<TC_I8S4>(P, A, T);
        default: return tc_prepare_t<TC_INT8>(P, A, T);
    }
}

template <int F>
static void launch_batch_t(const void *dargs, const int64_t *doff, int nplan, int64_t tiles, cudaStream_t s) {
    const size_t smem = tc_smem_bytes<F>();
    ensure_dyn_smem(k_m2l_tc_batch<F>, smem);
    k_m2l_tc_batch<F><<<(unsigned)tiles, TC_THREADS, smem, s>>>((const TcArgs *)dargs, doff, nplan);
    KIFMM_LAUNCHED();
}

void launch_m2l_tc_batch(int form, const void *dargs, const int64_t *doff, int nplan, int64_t tiles,
                         cudaStream_t s) {
    KIFMM_REQUIRE(tiles > 0 && tiles < (1ll << 31), KIFMM_ERR_ARG, "batch M2L: bad tile count");
    switch (form) {
        case TC_BF16: launch_batch_t<TC_BF16>(dargs, doff, nplan, tiles, s); break;
        case TC_FP16: launch_batch_t<TC_FP16>(dargs, doff, nplan, tiles, s); break;
        case TC_I8S4: launch_batch_t<TC_I8S4>(dargs, doff, nplan, tiles, s); break;
        default: launch_batch_t<TC_INT8>(dargs, doff, nplan, tiles, s); break;
    }
}

}  // namespace kifmm
