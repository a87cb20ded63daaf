// noalloc.cu -- Morton sort of points for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc: code that runs while
// another component owns all device memory (a host application with its own
// pool that forbids outside allocations), or a latency-bound loop that must
// not enter the allocator.  kifmm_morton_sort_noalloc gives them the first
// stage of the tree build -- exact Morton keys on the root box and the stable
// radix sort of the points -- with every scratch byte in one file-scope
// device array of fixed size.  The caller passes the inputs and the outputs.
#include <cmath>
#include <mutex>

#include "kifmm_internal.cuh"

namespace kifmm {

void launch_morton_keys(const double *x, const double *y, int64_t n, double m, double M, uint64_t *key,
                        int32_t *perm, unsigned long long *outside, int num_sms, cudaStream_t stream);
int64_t radix_sort_hist_words(int64_t n);
void radix_sort_pairs_scratch(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, uint32_t *hist,
                              int64_t n, int bits, cudaStream_t stream);

// Scratch layout: key ping-pong [NMAX] u64 | index ping-pong [NMAX] i32 |
// digit histograms, 256 words per radix tile plus 256 (radix_sort_hist_words).
// About 12.3 MB.
constexpr int64_t NA_MAX = KIFMM_NOALLOC_MAX_POINTS;
constexpr int64_t NA_HIST_WORDS = (int64_t)256 * ((NA_MAX + RADIX_TILE_KEYS - 1) / RADIX_TILE_KEYS) + 256;
constexpr size_t NA_KEY_OFF = 0;
constexpr size_t NA_IDX_OFF = NA_KEY_OFF + (size_t)NA_MAX * 8;
constexpr size_t NA_HIST_OFF = NA_IDX_OFF + (size_t)NA_MAX * 4;
constexpr size_t NA_BYTES = NA_HIST_OFF + (size_t)NA_HIST_WORDS * 4;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// Device address of the scratch array, looked up once per device (with that
// device current) and cached for the life of the process.  CUDA loads this
// file's module lazily by default, so the lookup is also what makes the array
// resident on the device: the first call on a device allocates its ~12.3 MB
// (CUDA_MODULE_LOADING=EAGER reserves it when the library loads instead).
// The cached address does not survive cudaDeviceReset.
static std::mutex g_na_mutex;
static void *g_na_ptr[64] = {};
static int g_na_sms[64] = {};

static unsigned char *noalloc_scratch(int device, int *sms) {
    KIFMM_REQUIRE(device >= 0 && device < 64, KIFMM_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[device]) {
        void *ptr = nullptr;
        KIFMM_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        int n = 0;
        KIFMM_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
        g_na_sms[device] = n > 0 ? n : 148;
        g_na_ptr[device] = ptr;
    }
    *sms = g_na_sms[device];
    return (unsigned char *)g_na_ptr[device];
}

void set_error(const std::string &msg);

}  // namespace kifmm

using namespace kifmm;

extern "C" int kifmm_morton_sort_noalloc(const double *x, const double *y, int64_t n, double root_min,
                                         double root_max, uint64_t *keys, int32_t *perm, void *stream) {
    try {
        set_error("");
        KIFMM_REQUIRE(n >= 1, KIFMM_ERR_ARG, "morton_sort_noalloc: need at least one point");
        KIFMM_REQUIRE(n <= NA_MAX, KIFMM_ERR_ARG,
                      "morton_sort_noalloc: n exceeds KIFMM_NOALLOC_MAX_POINTS (1048576), the size of the "
                      "library's fixed scratch array");
        KIFMM_REQUIRE(x && y && keys && perm, KIFMM_ERR_ARG, "morton_sort_noalloc: null pointer");
        KIFMM_REQUIRE(std::isfinite(root_min) && std::isfinite(root_max) && root_max > root_min, KIFMM_ERR_ARG,
                      "morton_sort_noalloc: need finite root_min < root_max");
        KIFMM_REQUIRE(std::floor(root_min) == root_min && std::floor(root_max) == root_max, KIFMM_ERR_ARG,
                      "morton_sort_noalloc: the root box corners are integers (as kifmm_get_tree_info reports)");
        KIFMM_REQUIRE(std::fabs(root_min) < 8388608.0 && std::fabs(root_max) < 8388608.0, KIFMM_ERR_RANGE,
                      "morton_sort_noalloc: |root box| must stay below 2^23");
        int device = 0;
        KIFMM_CUDA(cudaGetDevice(&device));
        int sms = 148;
        unsigned char *base = noalloc_scratch(device, &sms);
        cudaStream_t s = (cudaStream_t)stream;
        uint64_t *ktmp = (uint64_t *)(base + NA_KEY_OFF);
        int32_t *itmp = (int32_t *)(base + NA_IDX_OFF);
        uint32_t *hist = (uint32_t *)(base + NA_HIST_OFF);
        KIFMM_REQUIRE(radix_sort_hist_words(n) <= NA_HIST_WORDS, KIFMM_ERR_CUDA,
                      "morton_sort_noalloc: histogram table smaller than the sort needs");
        // every scratch word the sort reads is written by the same call first
        // (histograms are zeroed per pass), so nothing is cleared here
        launch_morton_keys(x, y, n, root_min, root_max, keys, perm, nullptr, sms, s);
        radix_sort_pairs_scratch(keys, perm, ktmp, itmp, hist, n, 2 * KEY_DEPTH, s);
        return KIFMM_OK;
    } catch (const Fail &e) {
        return e.code;
    } catch (...) {
        set_error("unexpected C++ exception");
        return KIFMM_ERR_CUDA;
    }
}
