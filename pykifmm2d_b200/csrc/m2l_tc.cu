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
// owns TC_N = 32 targets and one 128-row M tile (its five int8 accumulators
// fit a 256-column TMEM allocation and its tiles 101 KB of shared memory, so
// two CTAs share an SM and one's copies overlap the other's MMAs); per direction (and per
// K chunk of 128) it stages A and B in shared memory in the UMMA K-major,
// no-swizzle layout, one thread issues the MMA chain, tcgen05.commit signals
// an mbarrier, and the epilogue reads TMEM with tcgen05.ld.
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

enum TcForm { TC_INT8 = 0, TC_BF16 = 1, TC_FP16 = 2 };
template <int F> struct TcTraits;
template <> struct TcTraits<TC_INT8> { static constexpr int NS = 5, EB = 1, KSTEP = 32, NACC = 5, NCOLS = 256; };
template <> struct TcTraits<TC_BF16> { static constexpr int NS = 2, EB = 2, KSTEP = 16, NACC = 1, NCOLS = 32; };
template <> struct TcTraits<TC_FP16> { static constexpr int NS = 2, EB = 2, KSTEP = 16, NACC = 1, NCOLS = 32; };

constexpr int TC_M = 128;      // MMA M: operator rows per tile (TMEM lanes)
constexpr int TC_N = 32;       // MMA N: target groups per CTA
constexpr int TC_KC = 128;     // K elements staged per stage
// Stages in flight.  One: at K = 128 a stage is 100 KB, and two CTAs per SM
// (one's copies under the other's MMAs) measured faster than two 64-K slots in
// one CTA, whose extra stages cost more synchronisation than they hid.
constexpr int TC_SLOTS = 1;
constexpr int TC_THREADS = 128;
static_assert(TC_N % 16 == 0 && TC_N >= 16 && TC_N <= 256, "MMA N for M = 128");
static_assert(TcTraits<TC_INT8>::NACC * TC_N <= TcTraits<TC_INT8>::NCOLS, "int8 accumulators exceed the TMEM allocation");
static_assert(TcTraits<TC_BF16>::NACC * TC_N <= TcTraits<TC_BF16>::NCOLS, "accumulator exceeds the TMEM allocation");
static_assert(2 * TcTraits<TC_INT8>::NCOLS <= 512, "two CTAs per SM must fit the 512 TMEM columns");
constexpr double FP16_PRESCALE = 4096.0;

struct TcGeom {
    int Q4, MP, MT, KP, NKC;   // rows, padded rows, M tiles, padded K per direction, K chunks
    size_t slice_bytes;        // one slice of one A tile chunk: 128 x TC_KC x EB
    size_t level_bytes;        // all A slices of one level
};

template <int F>
static TcGeom tc_geom(int Q) {
    TcGeom g;
    g.Q4 = 4 * Q;
    g.MP = (g.Q4 + TC_M - 1) / TC_M * TC_M;
    g.MT = g.MP / TC_M;
    g.KP = (g.Q4 + TC_KC - 1) / TC_KC * TC_KC;
    g.NKC = g.KP / TC_KC;
    g.slice_bytes = (size_t)TC_M * TC_KC * TcTraits<F>::EB;
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
    uint32_t fmt = F == TC_INT8 ? ((2u << 4) | (1u << 7) | (1u << 10))    // s32 <- s8 x s8
                 : F == TC_BF16 ? ((1u << 4) | (1u << 7) | (1u << 10))    // f32 <- bf16 x bf16
                                : (1u << 4);                              // f32 <- f16 x f16
    return fmt | ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}
template <int F>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    if (F == TC_INT8) {
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
    if (F == TC_INT8) {
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
        int mt = r / TC_M, kc = k / TC_KC;
        unsigned char *tile = base + (((size_t)d * T.g.MT + mt) * T.g.NKC + kc) * TcTraits<F>::NS * sb;
        put_slices<F>(tile, sb, core_off(r % TC_M, k % TC_KC, TC_M, TcTraits<F>::EB), v);
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
    if (F == TC_INT8) {
        double m = 0.0;
        for (int c = lane; c < Q4; c += 32) m = fmax(m, fabs(u[c]));
        for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        int kg = 0;
        if (m > 0.0) {
            int e;
            frexp(m * (128.0 / 127.0), &e);  // m * 128/127 < 2^e
            kg = (e >= 0) ? (e + 6) / 7 : -((-e) / 7);
        }
        const double inv = ldexp(1.0, -7 * kg);
        for (int c = lane; c < T.KP; c += 32) {
            double r = c < Q4 ? u[c] * inv : 0.0;
#pragma unroll
            for (int i = 0; i < TR::NS; i++) {
                r *= 128.0;
                double q = rint(r);
                r -= q;
                ((int8_t *)out)[(size_t)i * T.KP + c] = (int8_t)q;
            }
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
__global__ void __launch_bounds__(TC_THREADS, 2) k_m2l_tc(TcArgs T) {
    using TR = TcTraits<F>;
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    pdl_trigger();
    pdl_wait();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const PassArgs &A = T.A;
    const int Q = A.Q, Q4 = T.g.Q4, KP = T.pre.KP;
    const size_t a_sb = T.g.slice_bytes;                       // A slice (128 x KC)
    const size_t b_sb = (size_t)TC_N * TC_KC * TR::EB;         // B slice (TC_N x KC)
    const size_t a_stage = TR::NS * a_sb, b_stage = TR::NS * b_sb;
    unsigned char *sA = tc_smem;                               // [TC_SLOTS][NS slices]
    unsigned char *sB = sA + TC_SLOTS * a_stage;               // [TC_SLOTS][NS slices]
    int *sgrp = (int *)(sB + TC_SLOTS * b_stage);              // [TC_N][9]
    int *sshift = sgrp + TC_N * 9;                             // [TC_N][9] slice shift (INT8)
    double *stau = (double *)(sshift + TC_N * 9 + 2);          // [TC_N]
    int *sact = (int *)(stau + TC_N);                          // [TC_N]
    uint64_t *bars = (uint64_t *)(sact + TC_N + 2);            // [0..1] A landed, [2..3] MMAs done (per stage slot)
    uint32_t *tslot = (uint32_t *)(bars + 4);

    // which level / column tile / M tile
    const int64_t tile = blockIdx.x;
    int l = T.lmin;
    while (l < T.lmax && T.tile_off[l + 1] <= tile) l++;
    const int64_t lt = tile - T.tile_off[l];
    const int mt = (int)(lt % T.g.MT);
    const int64_t ct = lt / T.g.MT;
    const int64_t ne = A.T.ne[l], eoff = A.T.eoff[l];
    const int64_t e0 = ct * TC_N;
    const int lt1 = l + 1;  // target level: its operators
    const unsigned char *alev = T.aslices + (size_t)lt1 * T.g.level_bytes;
    const double *rsl = T.rowscale + (size_t)lt1 * T.g.MP;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TR::NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid < TC_N) {
        int64_t e = e0 + tid;
        bool act = e < ne && !(A.ent[eoff + e] & 1);
        int p = act ? A.ent_node[eoff + e] : -1;
        int kcol = -1000000;
        for (int d = 0; d < 9; d++) {
            int grp = -1;
            if (act && d != 4) {
                grp = m2l_source_entry(A.ncoll, A.nent, A.nbot, A.ntop, p, d);
                if (F == TC_INT8 && grp >= 0) kcol = max(kcol, T.pre.gexp[grp]);
            }
            sgrp[tid * 9 + d] = grp;
        }
        if (kcol == -1000000) kcol = 0;
        for (int d = 0; d < 9; d++) {
            int grp = sgrp[tid * 9 + d];
            sshift[tid * 9 + d] = (F == TC_INT8 && grp >= 0) ? kcol - T.pre.gexp[grp] : 0;
        }
        stau[tid] = F == TC_INT8 ? ldexp(1.0, 7 * kcol) : 1.0;
        sact[tid] = act;
    }
    if (tid == 0)
        for (int i = 0; i < 4; i++) mbar_init(smem_u32(&bars[i]));
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = instr_desc<F>();
    const uint32_t bfull[2] = {smem_u32(&bars[0]), smem_u32(&bars[1])};
    const uint32_t bdone[2] = {smem_u32(&bars[2]), smem_u32(&bars[3])};
    uint32_t pfull[2] = {0u, 0u}, pdone[2] = {0u, 0u};
    int nfull[2] = {0, 0}, ndone[2] = {0, 0};  // copies / commits issued and not yet waited for, per slot
    bool failed = false;
    const uint32_t a_bytes = (uint32_t)a_stage;
    constexpr int CH = TC_KC * TR::EB / 16;  // 16-byte chunks per slice row
    const int NKC = T.g.NKC, NST = 8 * NKC;   // stages: (direction != centre, K chunk)

    // stage st into slot: A by one bulk copy (on bfull[slot]), B by 16-byte copies
    // of the pre-sliced source groups (shifted slices for INT8)
    auto prepare = [&](int st, int slot) {
        const int dd = st / NKC, d = dd < 4 ? dd : dd + 1, kc = st % NKC;
        if (tid == 0) {
            mbar_expect_tx(bfull[slot], a_bytes);
            bulk_g2s(smem_u32(sA + slot * a_stage), alev + (((size_t)d * T.g.MT + mt) * NKC + kc) * a_stage, a_bytes,
                     bfull[slot]);
        }
        nfull[slot]++;
        unsigned char *sBs = sB + slot * b_stage;
        // all of a thread's loads first, then its stores: one round trip per stage
        constexpr int NBI = TC_N * TR::NS * CH, NB = (NBI + TC_THREADS - 1) / TC_THREADS;
        uint4 v[NB];
#pragma unroll
        for (int q = 0; q < NB; q++) {
            const int idx = tid + q * TC_THREADS;
            v[q] = make_uint4(0, 0, 0, 0);
            if (idx < NBI) {
                const int c = idx % CH, i = (idx / CH) % TR::NS, j = idx / (CH * TR::NS);
                const int grp = sgrp[j * 9 + d], si = i - sshift[j * 9 + d];
                if (grp >= 0 && si >= 0 && si < TR::NS)
                    v[q] = __ldg((const uint4 *)(T.pre.slices + ((size_t)grp * TR::NS + si) * KP * TR::EB +
                                                 (size_t)kc * TC_KC * TR::EB + c * 16));
            }
        }
#pragma unroll
        for (int q = 0; q < NB; q++) {
            const int idx = tid + q * TC_THREADS;
            if (idx < NBI) {
                const int c = idx % CH, i = (idx / CH) % TR::NS, j = idx / (CH * TR::NS);
                *(uint4 *)(sBs + i * b_sb + core_off(j, c * 16 / TR::EB, TC_N, TR::EB)) = v[q];
            }
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
    };
    // bounded wait on a slot barrier, uniform over the block
    // (a wait that runs out is tried once more, bounded, so that a copy or MMA
    // still in flight lands before the block frees TMEM and leaves)
    auto wait_slot = [&](const uint32_t *bar, uint32_t *par, int *cnt, int slot) {
        bool ok = mbar_wait(bar[slot], par[slot], T.wait_limit);
        if (!ok) mbar_wait(bar[slot], par[slot], kDrainWaitPolls);
        par[slot] ^= 1u;
        cnt[slot]--;
        return __syncthreads_or(!ok) == 0;
    };

    // pipeline over TC_SLOTS slots: the MMAs of stage st run on the tensor pipe
    // while the block stages st + 1 into the next slot
    prepare(0, 0);
    for (int st = 0; st < NST && !failed; st++) {
        const int slot = st % TC_SLOTS;
        if (!wait_slot(bfull, pfull, nfull, slot)) {
            failed = true;
            break;
        }
        if (tid == 0) {
            fence_after();
            const uint32_t a0 = smem_u32(sA + slot * a_stage), b0 = smem_u32(sB + slot * b_stage);
            const uint32_t a_lbo = (TC_M / 8) * 128, b_lbo = (TC_N / 8) * 128;
            for (int ks = 0; ks < TC_KC / TR::KSTEP; ks++) {
                for (int i = 0; i < TR::NS; i++) {
                    const int jmax = F == TC_INT8 ? TR::NS - 1 - i : (i == 0 ? 1 : 0);
                    for (int jj = 0; jj <= jmax; jj++) {
                        const int acc = F == TC_INT8 ? i + jj : 0;
                        const bool first = st == 0 && ks == 0 && i == 0 && (F == TC_INT8 || jj == 0);
                        uint64_t ad = umma_desc(a0 + i * (uint32_t)a_sb + ks * 2 * a_lbo, a_lbo, 128);
                        uint64_t bd = umma_desc(b0 + jj * (uint32_t)b_sb + ks * 2 * b_lbo, b_lbo, 128);
                        mma_issue<F>(tmem + acc * TC_N, ad, bd, idesc, first ? 0u : 1u);
                    }
                }
            }
            mma_commit(bdone[slot]);
        }
        ndone[slot]++;
        if (st + 1 < NST) {
            const int ns = (st + 1) % TC_SLOTS;
            if (ndone[ns] > 0 && !wait_slot(bdone, pdone, ndone, ns)) {  // the MMAs that last read slot ns
                failed = true;
                break;
            }
            prepare(st + 1, ns);
        }
    }
    // drain what is still in flight (on failure too: copies must land and MMAs
    // finish before the block frees TMEM and leaves)
    for (int sl = 0; sl < TC_SLOTS; sl++) {
        while (ndone[sl] > 0)
            if (!wait_slot(bdone, pdone, ndone, sl)) failed = true;
        while (nfull[sl] > 0)
            if (!wait_slot(bfull, pfull, nfull, sl)) failed = true;
    }
    fence_after();

    if (!failed) {
        const int row = warp * 32 + lane, r = mt * TC_M + row;
        const double sig = rsl[r];
#pragma unroll 1
        for (int cc = 0; cc < TC_N / 16; cc++) {
            double y[16];
#pragma unroll
            for (int c = 0; c < 16; c++) y[c] = 0.0;
#pragma unroll 1
            for (int s = 0; s < TR::NACC; s++) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(s * TC_N + cc * 16), v);
                const double w = F == TC_INT8 ? ldexp(1.0, -7 * (s + 2))
                               : F == TC_FP16 ? 1.0 / FP16_PRESCALE : 1.0;
#pragma unroll
                for (int c = 0; c < 16; c++)
                    y[c] += (F == TC_INT8 ? (double)(int32_t)v[c] : (double)__uint_as_float(v[c])) * w;
            }
            if (r < Q4)
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    const int j = cc * 16 + c;
                    if (sact[j]) {
                        int64_t cg = A.T.off[lt1] + 4 * (e0 + j);
                        A.udown[(size_t)cg * Q + r] = y[c] * sig * stau[j];
                    }
                }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TR::NCOLS));
    }
    if (failed && tid == 0) atomicOr(T.err, 1ull);
}

// ------------------------------------------------------------ host side
bool uses_tensor_m2l(const kifmm_plan *P) {
    return P->opt.precision == KIFMM_PREC_MIXED &&
           (P->opt.m2l == KIFMM_M2L_INT8 || P->opt.m2l == KIFMM_M2L_BF16X3 || P->opt.m2l == KIFMM_M2L_FP16X3);
}

static int form_of(int m2l) {
    return m2l == KIFMM_M2L_BF16X3 ? TC_BF16 : m2l == KIFMM_M2L_FP16X3 ? TC_FP16 : TC_INT8;
}

template <int F>
static size_t tc_smem_bytes() {
    using TR = TcTraits<F>;
    return TC_SLOTS * (TR::NS * (size_t)TC_M * TC_KC * TR::EB + TR::NS * (size_t)TC_N * TC_KC * TR::EB) + 2 * TC_N * 9 * 4 +
           8 + TC_N * 8 + TC_N * 4 + 8 + 32 + 8 + 1024;
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
        default: build_tc_ops_t<TC_INT8>(P); break;
    }
}

template <int F>
static void run_m2l_tensor_t(kifmm_plan *P, const PassArgs &A) {
    using TR = TcTraits<F>;
    TcGeom g = tc_geom<F>(P->Q);
    const int L = P->L;
    if (L < 3 || !P->n_ent) return;
    TcPre pre{};
    pre.KP = g.KP;
    P->tc_pre.alloc((size_t)P->n_ent * TR::NS * g.KP * TR::EB);
    P->tc_gexp.alloc(P->n_ent);
    pre.slices = P->tc_pre.p;
    pre.gexp = P->tc_gexp.p;
    launch_pdl(k_tc_preslice<F>, dim3(grid_for(P->n_ent * 32, 256)), dim3(256), 0, P->stream, A, P->n_ent, pre);
    TcArgs T{};
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
        if (l >= T.lmin && l <= T.lmax) tiles += (P->lt.ne[l] + TC_N - 1) / TC_N * g.MT;
    }
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
        default: run_m2l_tensor_t<TC_INT8>(P, A); break;
    }
}

}  // namespace kifmm
