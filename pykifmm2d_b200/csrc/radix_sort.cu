// radix_sort.cu -- stable LSD radix sort of 64-bit keys (optionally with int32
// payloads) for the Morton-key tree build.
//
// The plan's sorts use the onesweep form further down (one histogram kernel,
// then one kernel per 8-bit digit).  The no-allocation entry point keeps the
// three-kernel form, whose scratch is a fixed histogram table: each pass
// sorts one 8-bit digit in three kernels:
//   1. per-tile digit histograms (tile = 256 threads x 16 keys),
//   2. a per-digit exclusive scan over the tiles (one block per digit), which
//      also leaves the 256 digit totals behind the table,
//   3. a stable scatter: inside a tile, each warp ranks its 512 keys in order
//      with __match_any_sync, warps are combined by a per-digit prefix in
//      shared memory, and the tile's base is the digit's start (a scan of the
//      digit totals) plus the digit's scanned tile prefix.
#include <algorithm>

#include "kifmm_internal.cuh"

namespace kifmm {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
static_assert(RS_TILE == RADIX_TILE_KEYS, "histogram tables sized outside this file assume RADIX_TILE_KEYS per tile");
constexpr int RS_WARPS = RS_THREADS / 32;

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint64_t *__restrict__ key, int64_t n, int shift,
                                                         uint32_t *__restrict__ hist, int nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int i = 0; i < RS_ITEMS; i++) {
        int64_t idx = base + i * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[(key[idx] >> shift) & 255], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Per-digit scan: block d turns hist[d][0..nb) into exclusive prefixes over
// the tiles and writes the digit's total to dtot[d] (dtot = hist + 256 * nb).
__global__ void __launch_bounds__(256) k_rs_scan(uint32_t *__restrict__ hist, int nblocks) {
    __shared__ uint32_t part[256];
    uint32_t *h = hist + (size_t)blockIdx.x * nblocks;
    const int chunk = (nblocks + 255) / 256;
    const int b = threadIdx.x * chunk, e = min(b + chunk, nblocks);
    uint32_t sum = 0;
    for (int i = b; i < e; i++) sum += h[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - sum;
    for (int i = b; i < e; i++) {
        uint32_t v = h[i];
        h[i] = run;
        run += v;
    }
    if (threadIdx.x == 255) hist[(size_t)256 * nblocks + blockIdx.x] = part[255];
}

template <bool PAIRS>
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint64_t *__restrict__ key, const int32_t *__restrict__ val,
                                                            uint64_t *__restrict__ okey, int32_t *__restrict__ oval,
                                                            int64_t n, int shift, const uint32_t *__restrict__ hist,
                                                            int nblocks) {
    __shared__ uint32_t wcnt[RS_WARPS][256];
    __shared__ uint32_t base[256];
    __shared__ uint32_t wsum[RS_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < 256 * RS_WARPS; d += RS_THREADS) (&wcnt[0][0])[d] = 0;
    {  // digit bases: exclusive scan of the 256 digit totals
        uint32_t t = hist[(size_t)256 * nblocks + threadIdx.x], x = t;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        uint32_t woff = 0;
        for (int i = 0; i < w; i++) woff += wsum[i];
        base[threadIdx.x] = woff + x - t + hist[(size_t)threadIdx.x * nblocks + blockIdx.x];
    }
    __syncthreads();
    const int64_t t0 = (int64_t)blockIdx.x * RS_TILE + (int64_t)w * (RS_ITEMS * 32);
    uint64_t k[RS_ITEMS];
    int32_t v[RS_ITEMS];
    uint32_t rank[RS_ITEMS];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        int64_t idx = t0 + r * 32 + lane;
        bool ok = idx < n;
        k[r] = ok ? key[idx] : 0;
        if (PAIRS) v[r] = ok ? val[idx] : 0;
        uint32_t d = ok ? (uint32_t)((k[r] >> shift) & 255) : 256u;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = d < 256 ? wcnt[w][d] : 0;
        rank[r] = before + __popc(peers & lt);
        __syncwarp();
        if (d < 256 && lane == __ffs(peers) - 1) wcnt[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps for each digit, folded into per-warp offsets
    {
        int d = threadIdx.x;
        uint32_t run = base[d];
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ww++) {
            uint32_t c = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        int64_t idx = t0 + r * 32 + lane;
        if (idx < n) {
            uint32_t d = (uint32_t)((k[r] >> shift) & 255);
            uint32_t pos = wcnt[w][d] + rank[r];
            okey[pos] = k[r];
            if (PAIRS) oval[pos] = v[r];
        }
    }
}

// ---------------------------------------------------------------- onesweep
// The plan's sorts: one read of the keys counts the digits of every pass
// (k_os_hist), then each pass is ONE kernel (k_os_pass) that ranks a tile's
// keys as k_rs_scatter does and finds the tile's offset for each digit by a
// look-back over the tiles before it: every tile publishes its digit counts as
// soon as it has ranked its keys; the tiles of a pass all run at once, so
// instead of a chain of inclusive prefixes (one round trip per 32 tiles) the
// look-back has two levels, tiles within a group of 32 and group totals.
// Tiles take their index from a counter in the order they start, so every
// tile waited on is already running and publishes without waiting on later
// tiles.  Waits are bounded; one that runs out sets *err (the build fails).
constexpr int OS_MAX_PASSES = 8;
struct OsShifts {
    int n;
    int s[OS_MAX_PASSES];
};
constexpr unsigned long long OS_AGG = 1ull << 62, OS_VAL = (1ull << 62) - 1;
constexpr int OS_GROUP = 32;  // tiles per look-back group

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// digit counts of every pass; shifts packed 8 bits each in `packed` (no
// per-pass array in local memory), npass <= OS_MAX_PASSES
__global__ void __launch_bounds__(RS_THREADS) k_os_hist(const uint64_t *__restrict__ key, int64_t n, uint64_t packed,
                                                         int npass, uint32_t *__restrict__ hist) {
    // warp-private counters per pass (conflicts only among a warp's own lanes):
    // dynamic shared memory [RS_WARPS][npass][256]
    extern __shared__ uint32_t h_dyn[];
    pdl_trigger();
    pdl_wait();
    for (int i = threadIdx.x; i < RS_WARPS * npass * 256; i += RS_THREADS) h_dyn[i] = 0;
    __syncthreads();
    const int w = threadIdx.x >> 5;
    for (int64_t base = (int64_t)blockIdx.x * RS_TILE; base < n; base += (int64_t)gridDim.x * RS_TILE) {
        uint64_t k[RS_ITEMS];
#pragma unroll
        for (int r = 0; r < RS_ITEMS; r++) {
            const int64_t idx = base + r * RS_THREADS + threadIdx.x;
            k[r] = idx < n ? key[idx] : 0;
        }
#pragma unroll
        for (int p = 0; p < OS_MAX_PASSES; p++) {
            if (p >= npass) break;
            const int sh = (int)((packed >> (8 * p)) & 63);
#pragma unroll
            for (int r = 0; r < RS_ITEMS; r++)
                if (base + r * RS_THREADS + threadIdx.x < n)
                    atomicAdd(&h_dyn[(w * npass + p) * 256 + ((k[r] >> sh) & 255)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npass * 256; i += RS_THREADS) {
        uint32_t c = 0;
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ww++) c += h_dyn[ww * npass * 256 + i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// One pass.  The tile's keys are ranked per warp, ordered by digit in shared
// memory (tile-local digit starts tstart[]), and written out in that order so
// that consecutive threads store consecutive positions of one digit's run.
// keys per thread in a onesweep tile (4096-key tiles, two CTAs per SM, every
// tile of a 1M-key pass resident at once); 4 and 8 keys per thread measured
// 2.2x slower on the 1M-point tree build (0.20 against 0.091 ms for the sort)
constexpr int OS_ITEMS = 16;
constexpr int OS_TILE = RS_THREADS * OS_ITEMS;
constexpr size_t OS_PASS_SMEM = (size_t)OS_TILE * (sizeof(uint64_t) + sizeof(int32_t));
template <bool PAIRS>
__global__ void __launch_bounds__(RS_THREADS) k_os_pass(const uint64_t *__restrict__ key, const int32_t *__restrict__ val,
                                                         uint64_t *__restrict__ okey, int32_t *__restrict__ oval,
                                                         int64_t n, int shift, const uint32_t *__restrict__ ghist,
                                                         unsigned long long *status, unsigned *tile_ctr,
                                                         unsigned long long *err, long long limit) {
    pdl_trigger();
    pdl_wait();
    extern __shared__ __align__(16) unsigned char os_sm[];
    uint64_t *skey = (uint64_t *)os_sm;                        // [OS_TILE]
    int32_t *sval = (int32_t *)(os_sm + OS_TILE * sizeof(uint64_t));
    __shared__ uint32_t wcnt[RS_WARPS][256];
    __shared__ uint32_t tstart[256];
    __shared__ uint32_t dbase[256];
    __shared__ uint32_t wsum[2][RS_WARPS];
    __shared__ unsigned tile_s;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_ctr, 1u);
    for (int d = threadIdx.x; d < 256 * RS_WARPS; d += RS_THREADS) (&wcnt[0][0])[d] = 0;
    __syncthreads();
    const unsigned tile = tile_s;
    const int64_t tbase = (int64_t)tile * OS_TILE;
    const int tn = (int)min((int64_t)OS_TILE, n - tbase);
    const int64_t t0 = tbase + (int64_t)w * (OS_ITEMS * 32);
    uint64_t k[OS_ITEMS];
    int32_t v[OS_ITEMS];
    uint32_t rank[OS_ITEMS];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < OS_ITEMS; r++) {
        const int64_t idx = t0 + r * 32 + lane;
        const bool ok = idx < n;
        k[r] = ok ? key[idx] : 0;
        if (PAIRS) v[r] = ok ? val[idx] : 0;
    }
#pragma unroll
    for (int r = 0; r < OS_ITEMS; r++) {
        const bool ok = t0 + r * 32 + lane < n;
        const uint32_t d = ok ? (uint32_t)((k[r] >> shift) & 255) : 256u;
        const unsigned peers = warp_match_digit(d);
        const uint32_t before = d < 256 ? wcnt[w][d] : 0;
        rank[r] = before + __popc(peers & lt);
        __syncwarp();
        if (d < 256 && lane == __ffs(peers) - 1) wcnt[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    const int d = threadIdx.x;
    uint32_t tot = 0;
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ww++) {
        const uint32_t c = wcnt[ww][d];
        wcnt[ww][d] = tot;
        tot += c;
    }
    // this tile's digit counts, for the look-back of the later tiles
    st_relaxed_u64(status + (size_t)tile * 256 + d, OS_AGG | tot);
    // block scans over the digits: tile-local starts, and the pass's global starts
    const uint32_t g = ghist[d];
    uint32_t xt = tot, xg = g;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t yt = __shfl_up_sync(0xffffffffu, xt, o), yg = __shfl_up_sync(0xffffffffu, xg, o);
        if (lane >= o) {
            xt += yt;
            xg += yg;
        }
    }
    if (lane == 31) {
        wsum[0][w] = xt;
        wsum[1][w] = xg;
    }
    __syncthreads();
    uint32_t wt = 0, wg = 0;
    for (int i = 0; i < w; i++) {
        wt += wsum[0][i];
        wg += wsum[1][i];
    }
    const uint32_t ts = wt + xt - tot;
    tstart[d] = ts;
    __syncthreads();
    // the tile in digit order into shared memory, before the look-back, so
    // that the look-back has the registers for wide batches
#pragma unroll
    for (int r = 0; r < OS_ITEMS; r++) {
        if (t0 + r * 32 + lane < n) {
            const uint32_t dd = (uint32_t)((k[r] >> shift) & 255);
            const uint32_t li = tstart[dd] + wcnt[w][dd] + rank[r];
            skey[li] = k[r];
            if (PAIRS) sval[li] = v[r];
        }
    }
    // Two-level look-back.  Tiles form groups of OS_GROUP: a tile sums the
    // counts of the earlier tiles of its group (one batch of loads); the last
    // tile of a group then publishes the group's total; a tile adds the totals
    // of the earlier groups (one batch per OS_GROUP groups).  Every wait is on a
    // tile with a smaller index, which started earlier and publishes without
    // waiting on later tiles.  Polls are bounded; one that runs out sets *err.
    const unsigned long long *gbase = status + (size_t)gridDim.x * 256;  // [groups][256] group totals
    const unsigned grp = tile / OS_GROUP, tin = tile % OS_GROUP;
    uint32_t excl_in = 0, excl = 0;
    bool ok = true;
    auto sum_published = [&](const unsigned long long *base, unsigned cnt, uint32_t &acc) {
        unsigned rem = cnt >= 32 ? 0xffffffffu : ((1u << cnt) - 1u);
        long long polls = 0;
        while (rem) {
            unsigned long long sv[OS_GROUP];
#pragma unroll
            for (int q = 0; q < OS_GROUP; q++) sv[q] = ((rem >> q) & 1u) ? ld_relaxed_u64(base + (size_t)q * 256 + d) : 0ull;
#pragma unroll
            for (int q = 0; q < OS_GROUP; q++)
                if (((rem >> q) & 1u) && (sv[q] & ~OS_VAL)) {
                    acc += (uint32_t)(sv[q] & OS_VAL);
                    rem &= ~(1u << q);
                }
            if (rem && ++polls > limit) {
                atomicOr(err, 1ull);
                return false;
            }
        }
        return true;
    };
    if (tin > 0) ok = sum_published(status + (size_t)grp * OS_GROUP * 256, tin, excl_in);
    if (tin == OS_GROUP - 1 || tile == gridDim.x - 1)
        st_relaxed_u64((unsigned long long *)gbase + (size_t)grp * 256 + d, OS_AGG | (excl_in + tot));
    for (unsigned g0 = 0; ok && g0 < grp; g0 += OS_GROUP)
        ok = sum_published(gbase + (size_t)g0 * 256, min((unsigned)OS_GROUP, grp - g0), excl);
    excl += excl_in;
    dbase[d] = wg + xg - g + excl - ts;  // global position = dbase[digit] + tile-local index
    // a look-back that ran out leaves the offsets unknown: write nothing (*err is set)
    if (__syncthreads_or(!ok)) return;
    for (int i = threadIdx.x; i < tn; i += RS_THREADS) {
        const uint64_t kk = skey[i];
        const uint32_t pos = dbase[(uint32_t)((kk >> shift) & 255)] + (uint32_t)i;
        okey[pos] = kk;
        if (PAIRS) oval[pos] = sval[i];
    }
}

// Sort by the 8-bit digits at the given shifts (ascending), stable.
static void os_run(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, const int *shifts,
                   int npass, kifmm_plan *P, bool pairs) {
    if (n <= 1 || npass == 0) return;
    KIFMM_REQUIRE(n < (1ll << 31), KIFMM_ERR_ARG, "radix sort: more than 2^31 keys");
    KIFMM_REQUIRE(npass <= OS_MAX_PASSES, KIFMM_ERR_ARG, "radix sort: too many passes");
    cudaStream_t s = P->stream;
    const int64_t ntiles = (n + OS_TILE - 1) / OS_TILE;
    OsShifts sh{};
    sh.n = npass;
    for (int p = 0; p < npass; p++) sh.s[p] = shifts[p];
    // scratch: digit counts [npass][256], tile counters [npass], look-back status
    // [npass][ntiles][256] (one pass's worth, cleared before each pass, when large)
    // per pass: the tiles' digit counts, then the groups' totals
    const size_t per_pass = (size_t)(ntiles + (ntiles + OS_GROUP - 1) / OS_GROUP) * 256;
    const bool all_at_once = (size_t)npass * per_pass * 8 <= ((size_t)64 << 20);
    const size_t nstat = all_at_once ? (size_t)npass * per_pass : per_pass;
    P->sort_hist.alloc((size_t)npass * 256 + npass);
    P->sort_status.alloc(nstat);
    uint32_t *hist = P->sort_hist.p;
    unsigned *ctr = P->sort_hist.p + (size_t)npass * 256;
    launch_fill(P, {{hist, (size_t)npass * 256 + npass, 0u}, {P->sort_status.p, 2 * nstat, 0u}});
    const unsigned hg = (unsigned)std::min<int64_t>(ntiles, (int64_t)P->num_sms * 4);
    uint64_t packed = 0;
    for (int p = 0; p < npass; p++) packed |= (uint64_t)(shifts[p] & 63) << (8 * p);
    const size_t hsm = (size_t)RS_WARPS * npass * 256 * sizeof(uint32_t);
    ensure_dyn_smem(k_os_hist, hsm);
    launch_pdl(k_os_hist, dim3(hg), dim3(RS_THREADS), hsm, s, (const uint64_t *)key, n, packed, npass, hist);
    uint64_t *ka = key, *kb = key_tmp;
    int32_t *va = val, *vb = val_tmp;
    unsigned long long *err = P->scal.p + KIFMM_SCAL_SORT_ERR;
    for (int p = 0; p < npass; p++) {
        unsigned long long *stat = P->sort_status.p + (all_at_once ? (size_t)p * per_pass : 0);
        if (!all_at_once && p > 0)
            KIFMM_CUDA(cudaMemsetAsync(stat, 0, per_pass * sizeof(unsigned long long), s));
        if (pairs) {
            ensure_dyn_smem(k_os_pass<true>, OS_PASS_SMEM);
            launch_pdl(k_os_pass<true>, dim3((unsigned)ntiles), dim3(RS_THREADS), OS_PASS_SMEM, s,
                       (const uint64_t *)ka, (const int32_t *)va, kb, vb, n, sh.s[p], (const uint32_t *)(hist + 256 * p),
                       stat, ctr + p, err, 1ll << 20);
        } else {
            ensure_dyn_smem(k_os_pass<false>, OS_PASS_SMEM);
            launch_pdl(k_os_pass<false>, dim3((unsigned)ntiles), dim3(RS_THREADS), OS_PASS_SMEM, s,
                       (const uint64_t *)ka, (const int32_t *)nullptr, kb, (int32_t *)nullptr, n, sh.s[p],
                       (const uint32_t *)(hist + 256 * p), stat, ctr + p, err, 1ll << 20);
        }
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != key) {
        KIFMM_CUDA(cudaMemcpyAsync(key, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        if (pairs) KIFMM_CUDA(cudaMemcpyAsync(val, va, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    }
}

static void rs_run(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, int bits,
                   kifmm_plan *P, bool pairs, int lo_bit = 0) {
    int shifts[OS_MAX_PASSES];
    const int passes = (bits + 7) / 8;
    for (int p = 0; p < passes; p++) shifts[p] = lo_bit + 8 * p;
    os_run(key, val, key_tmp, val_tmp, n, shifts, passes, P, pairs);
}

void radix_sort_pairs(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, int bits,
                      kifmm_plan *P) {
    rs_run(key, val, key_tmp, val_tmp, n, bits, P, true);
}

// sorts by bits [lo_bit, lo_bit + bits) only (stable)
void radix_sort_pairs_bits(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, int lo_bit,
                           int bits, kifmm_plan *P) {
    rs_run(key, val, key_tmp, val_tmp, n, bits, P, true, lo_bit);
}

void radix_sort_keys(uint64_t *key, uint64_t *key_tmp, int64_t n, int bits, kifmm_plan *P) {
    rs_run(key, nullptr, key_tmp, nullptr, n, bits, P, false);
}

// keys sorted by the digits at `shifts` only: the caller knows the other
// digits are equal for every key
void radix_sort_keys_shifts(uint64_t *key, uint64_t *key_tmp, int64_t n, const int *shifts, int npass,
                            kifmm_plan *P) {
    os_run(key, nullptr, key_tmp, nullptr, n, shifts, npass, P, false);
}

int64_t radix_sort_hist_words(int64_t n) { return (int64_t)256 * ((n + RS_TILE - 1) / RS_TILE) + 256; }

// Same passes as rs_run, on caller-provided scratch (histogram table of
// radix_sort_hist_words(n) words, ping-pong buffers of n entries); launches
// only, no allocation.  `bits` must give an even number of passes so the
// result ends in key/val.
void radix_sort_pairs_scratch(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, uint32_t *hist,
                              int64_t n, int bits, cudaStream_t stream) {
    if (n <= 1) return;
    int nb = (int)((n + RS_TILE - 1) / RS_TILE);
    int passes = (bits + 7) / 8;
    uint64_t *ka = key, *kb = key_tmp;
    int32_t *va = val, *vb = val_tmp;
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        k_rs_hist<<<nb, RS_THREADS, 0, stream>>>(ka, n, shift, hist, nb);
        KIFMM_LAUNCHED();
        k_rs_scan<<<256, 256, 0, stream>>>(hist, nb);
        KIFMM_LAUNCHED();
        k_rs_scatter<true><<<nb, RS_THREADS, 0, stream>>>(ka, va, kb, vb, n, shift, hist, nb);
        KIFMM_LAUNCHED();
        uint64_t *tk = ka; ka = kb; kb = tk;
        int32_t *tv = va; va = vb; vb = tv;
    }
}

}  // namespace kifmm
