// draws.cu -- device-side densities and potential sums for serving.
//
// A serving request applies its plan to a sequence of fresh N(0,1) densities
// (the iterates of an iterative solve).  Density `index` of a request with
// seed `seed` is drawn here from a counter-based generator, so the numbers do
// not depend on which launch, stream or batch draws them: element 2j and
// 2j+1 come from one Philox4x32-10 block (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011) with counter
// (j, index) and key seed, turned into two normals by the Box-Muller
// transform (Box and Muller, 1958).
#include "kifmm_internal.cuh"

namespace kifmm {

struct DrawLane {
    double *out;     // the lane's density (n doubles)
    int64_t n;
    uint64_t seed;   // kDrawSkip: the caller writes the density
    uint64_t index;  // density number
};
constexpr uint64_t kDrawSkip = ~0ull;

// Philox4x32: ten rounds of two 32x32->64 multiplies per round with the
// multipliers and key increments of the paper's 4x32 variant.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// uniform double in (0, 1] from 64 random bits (53 of them used)
__device__ __forceinline__ double unit_open0(uint32_t a, uint32_t b) {
    const uint64_t m = (((uint64_t)a << 32) | b) >> 11;
    return ((double)m + 1.0) * 0x1.0p-53;
}

__device__ __forceinline__ void draw_pair(uint64_t seed, uint64_t index, int64_t j, double &z0, double &z1) {
    const uint4 c = make_uint4((uint32_t)j, (uint32_t)((uint64_t)j >> 32), (uint32_t)index, (uint32_t)(index >> 32));
    const uint4 r = philox4x32_10(c, make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const double u1 = unit_open0(r.x, r.y), u2 = unit_open0(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    z0 = rad * co;
    z1 = rad * s;
}

__device__ __forceinline__ void fill_lane(const DrawLane &L, int64_t first, int64_t stride) {
    const int64_t pairs = (L.n + 1) >> 1;
    for (int64_t j = first; j < pairs; j += stride) {
        double z0, z1;
        draw_pair(L.seed, L.index, j, z0, z1);
        L.out[2 * j] = z0;
        if (2 * j + 1 < L.n) L.out[2 * j + 1] = z1;
    }
}

__global__ void k_fill_normal(DrawLane L) {
    fill_lane(L, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// every lane of a batch: blockIdx.y is the lane
__global__ void k_fill_normal_lanes(const DrawLane *__restrict__ lanes) {
    const DrawLane L = lanes[blockIdx.y];
    if (L.seed == kDrawSkip) return;
    fill_lane(L, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// sums[r] = sum of lane r's potentials, one block per lane in a fixed order
constexpr int SUM_THREADS = 256;
__global__ void __launch_bounds__(SUM_THREADS) k_lane_sums(const DrawLane *__restrict__ lanes,
                                                           double *__restrict__ sums) {
    __shared__ double red[SUM_THREADS / 32];
    const DrawLane L = lanes[blockIdx.x];
    double v = 0.0;
    for (int64_t i = threadIdx.x; i < L.n; i += SUM_THREADS) v += L.out[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < SUM_THREADS / 32; w++) t += red[w];
        sums[blockIdx.x] = t;
    }
}

static unsigned draw_blocks(int64_t n) {
    const int64_t pairs = (n + 1) / 2;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((pairs + 255) / 256, 4096));
}

void launch_fill_normal(double *out, int64_t n, uint64_t seed, uint64_t index, cudaStream_t s) {
    if (n <= 0) return;
    k_fill_normal<<<draw_blocks(n), 256, 0, s>>>(DrawLane{out, n, seed, index});
    KIFMM_LAUNCHED();
}

void launch_fill_lanes(const void *dlanes, int nlanes, int64_t nmax, cudaStream_t s) {
    KIFMM_REQUIRE(nlanes > 0 && nlanes <= 65535, KIFMM_ERR_ARG, "draws: bad lane count");
    k_fill_normal_lanes<<<dim3(draw_blocks(nmax), (unsigned)nlanes), 256, 0, s>>>((const DrawLane *)dlanes);
    KIFMM_LAUNCHED();
}

void launch_lane_sums(const void *dlanes, int nlanes, double *sums, cudaStream_t s) {
    k_lane_sums<<<(unsigned)nlanes, SUM_THREADS, 0, s>>>((const DrawLane *)dlanes, sums);
    KIFMM_LAUNCHED();
}

size_t draw_lane_bytes() { return sizeof(DrawLane); }

void set_draw_lane(void *lanes, int r, double *out, int64_t n, uint64_t seed, uint64_t index) {
    ((DrawLane *)lanes)[r] = DrawLane{out, n, seed, index};
}

void set_draw_seed(void *lanes, int r, uint64_t seed, uint64_t index) {
    ((DrawLane *)lanes)[r].seed = seed;
    ((DrawLane *)lanes)[r].index = index;
}

}  // namespace kifmm
