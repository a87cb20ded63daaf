// radix_sort.cu -- stable LSD radix sort of 64-bit keys (optionally with int32
// payloads) for the Morton-key tree build.
//
// Each pass sorts one 8-bit digit in three kernels:
//   1. per-tile digit histograms (tile = 256 threads x 16 keys),
//   2. a per-digit exclusive scan over the tiles (one block per digit), which
//      also leaves the 256 digit totals behind the table,
//   3. a stable scatter: inside a tile, each warp ranks its 512 keys in order
//      with __match_any_sync, warps are combined by a per-digit prefix in
//      shared memory, and the tile's base is the digit's start (a scan of the
//      digit totals) plus the digit's scanned tile prefix.
#include "kifmm_internal.cuh"

namespace kifmm {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
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

static void rs_run(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, int bits,
                   kifmm_plan *P, bool pairs, int lo_bit = 0) {
    if (n <= 1) return;
    KIFMM_REQUIRE(n < (1ll << 31), KIFMM_ERR_ARG, "radix sort: more than 2^31 keys");
    int nb = (int)((n + RS_TILE - 1) / RS_TILE);
    P->sort_hist.alloc((size_t)256 * nb + 256);
    int passes = (bits + 7) / 8;
    uint64_t *ka = key, *kb = key_tmp;
    int32_t *va = val, *vb = val_tmp;
    for (int p = 0; p < passes; p++) {
        int shift = lo_bit + 8 * p;
        k_rs_hist<<<nb, RS_THREADS, 0, P->stream>>>(ka, n, shift, P->sort_hist.p, nb);
        KIFMM_LAUNCHED();
        k_rs_scan<<<256, 256, 0, P->stream>>>(P->sort_hist.p, nb);
        KIFMM_LAUNCHED();
        if (pairs)
            k_rs_scatter<true><<<nb, RS_THREADS, 0, P->stream>>>(ka, va, kb, vb, n, shift, P->sort_hist.p, nb);
        else
            k_rs_scatter<false><<<nb, RS_THREADS, 0, P->stream>>>(ka, nullptr, kb, nullptr, n, shift,
                                                                  P->sort_hist.p, nb);
        KIFMM_LAUNCHED();
        uint64_t *tk = ka; ka = kb; kb = tk;
        int32_t *tv = va; va = vb; vb = tv;
    }
    if (ka != key) {
        KIFMM_CUDA(cudaMemcpyAsync(key, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, P->stream));
        if (pairs) KIFMM_CUDA(cudaMemcpyAsync(val, va, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, P->stream));
    }
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
