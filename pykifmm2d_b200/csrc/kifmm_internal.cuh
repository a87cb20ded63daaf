// kifmm_internal.cuh -- shared definitions of the sm_100a KIFMM library.
#pragma once
#include <initializer_list>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <utility>
#include <vector>

#include "kifmm2d.h"  // include/ (on the include path)

// ----------------------------------------------------------------- errors
namespace kifmm {

void set_error(const std::string &msg);

struct Fail {
    int code;
};

#define KIFMM_CUDA(call)                                                            \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            kifmm::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));  \
            throw kifmm::Fail{e_ == cudaErrorMemoryAllocation ? KIFMM_ERR_NOMEM     \
                                                              : KIFMM_ERR_CUDA};    \
        }                                                                           \
    } while (0)

#define KIFMM_REQUIRE(cond, code, msg)          \
    do {                                        \
        if (!(cond)) {                          \
            kifmm::set_error(msg);              \
            throw kifmm::Fail{code};            \
        }                                       \
    } while (0)

// Kernels launched by this library in the process (kifmm_launch_count).
extern std::atomic<long long> g_launch_count;

// Launch check: configuration errors surface at once, faults at the next sync.
#define KIFMM_LAUNCHED()                                                  \
    do {                                                                  \
        kifmm::g_launch_count.fetch_add(1, std::memory_order_relaxed);    \
        KIFMM_CUDA(cudaGetLastError());                                   \
    } while (0)

// ---------------------------------------------------------- device buffers
// Stream on which the current entry point orders its work; device buffers
// are allocated and freed stream-ordered on it (cudaMallocAsync from the
// device's default pool, which keeps freed blocks cached, see capi.cu).
extern thread_local cudaStream_t g_stream;

// A device allocation owned by a plan (freed by the plan's destructor).
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        void *q = nullptr;
        KIFMM_CUDA(cudaMallocAsync(&q, (count ? count : 1) * sizeof(T), g_stream));
        p = (T *)q;
        n = count;
        s = g_stream;
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    ~DBuf() { release(); }
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
};

// ---------------------------------------------------------- tree constants
// Points are keyed on a 2^D x 2^D grid over the root box; a level-l cell key
// is the top 2l bits of the 2D-bit Morton key (child order (hx, hy) -> 2hx+hy,
// the reference's (lo-x,lo-y), (lo-x,hi-y), (hi-x,lo-y), (hi-x,hi-y), tree.py:170-185).
constexpr int KEY_DEPTH = 29;
// Keys per tile of the plain LSD radix sort (radix_sort.cu: 256 threads x 16
// keys); callers that size its histogram table themselves use it.
constexpr int RADIX_TILE_KEYS = 4096;
// Taylor order of the Laplace L2P fast path (|z|/r2 <= 0.585 inside 0.75 w)
#define KIFMM_TAYLOR_P 48
constexpr int MAX_LEVELS = KIFMM_MAX_LEVELS;  // levels 0..29
// Split/X-list cell entries: (level << 57) | (cell key << 1) | is_xlist
constexpr int ENT_LEVEL_SHIFT = 57;
constexpr uint64_t ENT_EMPTY = ~0ull;

enum NodeFlags : uint8_t {
    NF_SPLIT = 1,   // real node that has real children (reference: not leaf, not fake)
    NF_XLIST = 2,   // real leaf split into fake children (reference Level.Xlist)
    NF_FAKE = 4,    // fake leaf (reference Level.fake_leaf)
};

struct LevelInfo {
    int64_t off;    // first global node index of the level
    int64_t n;      // nodes on the level
    int64_t eoff;   // first entry (split/X-list cell) of the level in the sorted list
    int64_t ne;     // entries on the level
    double width;
};

// Per-level geometry passed by value to kernels.
struct LevelTable {
    int L;
    int64_t off[MAX_LEVELS + 1];
    int64_t eoff[MAX_LEVELS + 1];
    int64_t ne[MAX_LEVELS + 1];
};

// Operator block of one level (device pointers into Plan::ops).
struct LevelOps {
    double *inv;    // [Q x Q]      check -> equivalent (E2C^-1)
    double *m2m;    // [Q x 4Q]     u_up(parent) = m2m . u_up(children)   (M2MC . Inv_{l+1})
    double *l2lT;   // [Q x 4Q]     transposed: u_down(children) = l2lT^T . u_down(parent)
    double *m2lT;   // [8][4Q x 4Q] transposed directional M2L blocks (CM2L . Inv)
    double *large;  // [2Q]         check-circle offsets (x then y)
    double *small;  // [2Q]         equivalent-circle offsets
};

struct PendingPhase {
    int id;
    cudaEvent_t a, b;
    long long launches;
};

}  // namespace kifmm

// --------------------------------------------------------------- the plan
struct kifmm_plan {
    // configuration
    kifmm_kernel kern{};
    int Q = 0;            // state length per node: Nequiv (real kernels), 2 Nequiv (complex: real, imaginary)
    int Qc = 0;           // points per circle (Nequiv)
    bool cplx = false;    // complex kernel: densities, potentials and check potentials complex
    int ppl = 0;          // Ncutoff
    kifmm_options opt{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // operator construction runs on a side stream of the plan while the tree
    // build continues (it needs only the root width and the depth); the main
    // stream waits on ops_done before the operators are used
    cudaStream_t side = nullptr;
    // the near field at the sources, started by build_expansions on a stream
    // of its own so that it runs under the far-field chain (mixed form)
    cudaStream_t near_stream = nullptr;  // lowest priority
    cudaEvent_t near_fork = nullptr, near_done = nullptr;
    // ... while the far-field chain runs on a stream of the highest priority,
    // so that its small launches are scheduled ahead of the near pass's blocks
    cudaStream_t far_stream = nullptr;
    cudaEvent_t far_fork = nullptr, far_done = nullptr;
    bool near_pending = false;  // P->pots holds the near field of the last apply, far field not added yet
    cudaEvent_t ops_fork = nullptr, ops_done = nullptr;
    cudaEvent_t ops_circ = nullptr;  // side stream: the check circles are written (the P2M's only operator input)
    cudaEvent_t tree_ev = nullptr;   // build_tree: the split-cell counts are on the host
    uint64_t spec_cap = 0;           // split-cell capacity for the next build (from the last one)
    bool ops_pending = false;
    bool ops_wait = false;  // operators joined by precompute, the main stream's wait for them not issued yet
    bool circ_wait = false; // ... and its wait for the check circles (ops_circ) not issued yet
    cudaGraphExec_t graph = nullptr;  // captured apply (kifmm_graph_capture)
    long long wait_limit = -1;        // poll budget of the apply kernels' first waits (-1: kDefaultWaitPolls)
    int device = 0;
    int num_sms = 148;

    // points
    int64_t N = 0;
    double root_min = 0, root_max = 0, W = 0;
    int64_t n_outside = 0;
    kifmm::DBuf<double> x, y;        // caller order
    kifmm::DBuf<double> xs, ys;      // Morton order
    kifmm::DBuf<uint64_t> pkey;      // sorted point keys
    kifmm::DBuf<int32_t> perm;       // sorted position -> caller index

    // tree
    bool have_tree = false;
    int L = 0;
    kifmm::LevelInfo lv[kifmm::MAX_LEVELS + 1]{};
    kifmm::LevelTable lt{};
    int64_t n_nodes = 0, n_ent = 0;
    kifmm::DBuf<uint64_t> ent;       // sorted entries
    kifmm::DBuf<int32_t> ent_node;   // entry -> node
    kifmm::DBuf<uint64_t> nkey;      // node cell key
    kifmm::DBuf<int8_t> nlev;        // node level
    kifmm::DBuf<uint8_t> nflag;      // NodeFlags
    kifmm::DBuf<int32_t> nbot, ntop; // point range (Morton order)
    kifmm::DBuf<int32_t> nparent, nchild, nent;  // parent, first child, own entry
    kifmm::DBuf<int32_t> ncoll;      // [n_nodes][9] colleagues by direction (dx+1)*3+(dy+1)
    kifmm::DBuf<int32_t> leaf_list, p2m_list;
    kifmm::DBuf<int32_t> leaf_rec;   // [n_leaf_list][32] leaf records (passes.cuh, LeafRec)
    kifmm::DBuf<int32_t> m2l_perm;   // [n_ent] M2L target order of the entries (build_m2l_order)
    kifmm::DBuf<int32_t> leaf_split; // leaves of more than 32 points (split leaf pass)
    kifmm::DBuf<uint16_t> m2l_key;   // [n_ent] direction mask of each entry (256: not split)
    kifmm::DBuf<int32_t> m2l_src8;   // [n_ent][8] source entry per direction (-1: none)
    kifmm::DBuf<unsigned> m2l_hist;  // [MAX_LEVELS + 1][257] counts, then cursors
    kifmm::DBuf<uint32_t> list_tiles;
    int64_t n_leaf_list = 0, n_p2m_list = 0;
    int64_t leaf_loff[KIFMM_MAX_LEVELS + 1] = {};  // leaf_list range of each level
    int64_t n_leaves = 0, n_fake = 0, n_xlist = 0;
    int64_t n_p2p_pairs = 0, n_p2m_points = 0, n_m2l_pairs = 0, n_m2l_groups = 0;
    bool have_stats = false;

    // operators
    bool have_ops = false;
    kifmm::DBuf<double> ops, ops_tmp;
    kifmm::LevelOps lops[kifmm::MAX_LEVELS + 1]{};
    kifmm::DBuf<float> ops_f;        // FP32 copies for the mixed passes
    kifmm::DBuf<uint16_t> ops_h;     // split half-precision M2L operators
    size_t ops_stride = 0;           // doubles per level block
    kifmm::DBuf<unsigned char> tc_a; // tensor-core M2L operator slices
    kifmm::DBuf<double> tc_rowscale;
    kifmm::DBuf<unsigned long long> tc_rowmax;  // [L][4Q] largest |value| per M2L operator row
    kifmm::DBuf<double> l2p_taylor;  // Laplace: [L][Q][2p+1] check potential -> Taylor coefficients
    kifmm::DBuf<double> leaf_coef;   // [n_leaf_list][2p+1] Taylor coefficients per apply
    kifmm::DBuf<unsigned char> tc_pre;  // per-apply slices of the source groups
    kifmm::DBuf<int> tc_gexp;
    // planned applies (planned.cu): P2M, L2P and near-field blocks, built on
    // the first apply after build_tree / precompute
    bool have_mats = false;
    size_t pm_bytes = 0;
    kifmm::DBuf<int64_t> pm_near_off, pm_l2p_off, pm_p2m_off;
    kifmm::DBuf<float> pm_near32;
    kifmm::DBuf<double> pm_near64, pm_l2p, pm_p2m;

    // workspaces
    kifmm::DBuf<double> tau, taus, pots, pot_out, tx, ty, tpot;
    // separate targets (evaluate_to_points): Morton-sorted copies, their order, and
    // the equivalent densities of the leaves' local expansions
    kifmm::DBuf<uint64_t> tkey, tkey2;
    kifmm::DBuf<int32_t> tperm, tperm2;
    kifmm::DBuf<double> txs, tys, node_den;
    kifmm::DBuf<double> uup, udown;
    kifmm::DBuf<double> zero4q;      // 4Q zeros: the source of an absent M2L direction
    bool have_expansions = false;
    bool applied = false;  // an apply at the sources ran since the tree / operators were built

    // scratch for the tree build
    kifmm::DBuf<uint64_t> key2, hash, list;
    uint64_t hash_cap = 1;            // slots of the split-cell hash table (power of two)
    kifmm::DBuf<int32_t> hash_idx;    // [hash_cap] sorted entry index of the entry in each slot
    kifmm::DBuf<int32_t> perm2;
    kifmm::DBuf<uint32_t> sort_hist;
    kifmm::DBuf<unsigned long long> sort_status;  // radix sort look-back words
    kifmm::DBuf<unsigned long long> scal;  // small device scalars
    kifmm::DBuf<int64_t> misc;
    // pinned host words (kifmm::HP_*): read-backs land here by asynchronous
    // copies followed by one stream sync (a copy to pageable memory would
    // block the host on every call), and the constant source of scal's reset
    unsigned long long *hpin = nullptr;

    // phase timers (kifmm_set_profiling)
    bool profiling = false;
    double phase_ms[KIFMM_PHASE_COUNT] = {};
    int64_t phase_launches[KIFMM_PHASE_COUNT] = {};
    std::vector<kifmm::PendingPhase> pending;
};

namespace kifmm {
// Brackets one phase with CUDA events on the plan's stream when profiling.
// Programmatic dependent launch: a kernel launched with launch_pdl may be
// scheduled while the previous kernel on the stream is still finishing; it
// calls pdl_wait() before it reads anything that kernel wrote (the wait
// returns once that grid has completed and its writes are visible), and
// pdl_trigger() to let the next one be scheduled.  Without the attribute both
// are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Fill ranges of 32-bit words with a value in one launch (programmatic
// dependent launch: it waits for the previous kernel before writing).  Used
// in place of chains of cudaMemsetAsync, each of which is a launch of its own
// that the next kernel cannot overlap.
struct FillRange {
    void *p;
    size_t words;
    uint32_t value;
};
void launch_fill(kifmm_plan *P, std::initializer_list<FillRange> ranges);
constexpr int M2L_KEYS = 257;  // direction-mask groups per level in the M2L target order (256 masks + non-split)
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    KIFMM_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
    KIFMM_LAUNCHED();
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device; the driver call is made once per (device, kernel, larger
// size), not before every launch.
void ensure_dyn_smem(const void *fn, size_t bytes);
template <class K>
inline void ensure_dyn_smem(K *fn, size_t bytes) {
    ensure_dyn_smem((const void *)fn, bytes);
}

// layout of kifmm_plan::hpin (64-bit words)
constexpr int HP_SCAL = 0;     // [16] snapshot of scal
constexpr int HP_MISC = 16;    // [128] snapshot of misc
constexpr int HP_INIT = 160;   // [16] reset values of scal (min trackers at ~0)
constexpr int HP_FLAGS = 192;  // [2] pass / tensor-core error flags
constexpr int HP_STATS = 200;  // [4] work counts
constexpr int HP_WORDS = 256;
unsigned long long *pinned_acquire();
void pinned_release(unsigned long long *p);

// Poll budgets of the bounded waits in the apply kernels: a first wait gets
// the plan's budget (kifmm_set_wait_limit, default kDefaultWaitPolls); if it
// runs out, the kernel flags the error and waits once more with
// kDrainWaitPolls so that its copies and MMAs in flight land before it frees
// its resources and returns.
constexpr long long kDefaultWaitPolls = 1ll << 26;
constexpr long long kDrainWaitPolls = 1ll << 26;
inline long long plan_wait_polls(const kifmm_plan *P) {
    return P->wait_limit >= 0 ? P->wait_limit : kDefaultWaitPolls;
}

// device scalar slots (plan->scal) holding error flags that the host reads
// after an apply: a bulk-copy wait in the level passes that ran out, and an
// MMA completion wait in the tensor-core M2L that ran out
constexpr int KIFMM_SCAL_SORT_ERR = 13;  // a radix-sort look-back wait that ran out
constexpr int KIFMM_SCAL_PASS_ERR = 14;
constexpr int KIFMM_SCAL_TC_ERR = 15;
constexpr int KIFMM_SCAL_LEAF_SPLIT = 16;  // count of the split leaf list (k_leaf_split_list)
constexpr int KIFMM_SCAL_WORDS = 17;

// Lanes of the warp holding the same 8-bit digit d (d = 256: no key; such
// lanes match each other only): nine ballots, one per bit, each lane keeping
// the lanes that agree with it on every bit.  All 32 lanes must call it.
// __match_any_sync gives the same mask, but its throughput falls with the
// number of distinct values in the warp, which for radix digits is high.
__device__ __forceinline__ unsigned warp_match_digit(uint32_t d) {
    unsigned m = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 9; b++) {
        const bool bit = (d >> b) & 1u;
        const unsigned bb = __ballot_sync(0xffffffffu, bit);
        m &= bit ? bb : ~bb;
    }
    return m;
}

struct PhaseScope {
    kifmm_plan *P;
    int id;
    cudaEvent_t a = nullptr;
    long long l0 = 0;
    PhaseScope(kifmm_plan *p, int phase);
    ~PhaseScope();
};
}  // namespace kifmm

// ------------------------------------------------------- kernel functions
namespace kifmm {

#include "k0_tables.h"

__device__ __forceinline__ double k0_d(double x) {
    if (x <= 2.0) {
        double t = x * x, a = K0_I0_D[K0_I0_D_N - 1], b = K0_P_D[K0_P_D_N - 1];
#pragma unroll
        for (int i = K0_I0_D_N - 2; i >= 0; i--) a = fma(a, t, K0_I0_D[i]);
#pragma unroll
        for (int i = K0_P_D_N - 2; i >= 0; i--) b = fma(b, t, K0_P_D[i]);
        return b - log(0.5 * x) * a;
    }
    double u = 4.0 / x - 1.0, b0 = 0.0, b1 = 0.0, b2;
#pragma unroll
    for (int i = K0_CHEB_D_N - 1; i >= 1; i--) {
        b2 = b1;
        b1 = b0;
        b0 = fma(2.0 * u, b1, K0_CHEB_D[i] - b2);
    }
    double f = fma(u, b0, K0_CHEB_D[0] - b1);
    return exp(-x) * rsqrt(x) * f;
}

__device__ __forceinline__ float k0_f(float x) {
    if (x <= 2.0f) {
        float t = x * x, a = K0_I0_F[K0_I0_F_N - 1], b = K0_P_F[K0_P_F_N - 1];
#pragma unroll
        for (int i = K0_I0_F_N - 2; i >= 0; i--) a = fmaf(a, t, K0_I0_F[i]);
#pragma unroll
        for (int i = K0_P_F_N - 2; i >= 0; i--) b = fmaf(b, t, K0_P_F[i]);
        return b - logf(0.5f * x) * a;
    }
    float u = 4.0f / x - 1.0f, b0 = 0.0f, b1 = 0.0f, b2;
#pragma unroll
    for (int i = K0_CHEB_F_N - 1; i >= 1; i--) {
        b2 = b1;
        b1 = b0;
        b0 = fmaf(2.0f * u, b1, K0_CHEB_F[i] - b2);
    }
    float f = fmaf(u, b0, K0_CHEB_F[0] - b1);
    return expf(-x) * rsqrtf(x) * f;
}

// G(r^2) for the plug-in kernels, FP64: Laplace -log(r^2)/(4 pi), modified
// Helmholtz K0(k r)/(2 pi).
__device__ __forceinline__ double green_d(int kind, double k, double r2) {
    if (kind == KIFMM_KERNEL_LAPLACE) return -0.07957747154594767 * log(r2);
    return 0.15915494309189535 * k0_d(k * sqrt(r2));
}
// Helmholtz kernel G = (i/4) H0^(1)(k r) = -Y0(k r)/4 + i J0(k r)/4, FP64
// (examples/hankel.py:37-39); (re, im).
__device__ __forceinline__ double2 green_c(double k, double r2) {
    const double z = k * sqrt(r2);
    return make_double2(-0.25 * y0(z), 0.25 * j0(z));
}
// value of a kernel as a complex number (the real kernels with zero imaginary part)
__device__ __forceinline__ double2 green_z(int kind, double k, double r2) {
    if (kind == KIFMM_KERNEL_HELMHOLTZ) return green_c(k, r2);
    return make_double2(green_d(kind, k, r2), 0.0);
}
__device__ __forceinline__ float green_f(int kind, float k, float r2) {
    if (kind == KIFMM_KERNEL_LAPLACE) return -0.0795774715f * __logf(r2);
    return 0.159154943f * k0_f(k * sqrtf(r2));
}

// Morton helpers (interleave with the x bit above the y bit)
__host__ __device__ __forceinline__ uint64_t spread2(uint64_t v) {
    v &= 0x00000000FFFFFFFFull;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}
__host__ __device__ __forceinline__ uint64_t compact2(uint64_t v) {
    v &= 0x5555555555555555ull;
    v = (v | (v >> 1)) & 0x3333333333333333ull;
    v = (v | (v >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v >> 4)) & 0x00FF00FF00FF00FFull;
    v = (v | (v >> 8)) & 0x0000FFFF0000FFFFull;
    v = (v | (v >> 16)) & 0x00000000FFFFFFFFull;
    return v;
}
__host__ __device__ __forceinline__ uint64_t morton(uint64_t ix, uint64_t iy) {
    return (spread2(ix) << 1) | spread2(iy);
}

// Source of the M2L from direction d of parent p: the entry (split or X-list
// cell) of the colleague in that direction, -1 when there is none, when it has
// no children, or when its children hold no points (their check potentials
// are zero; the reference skips such groups through parent_density_ind,
// class_fmm.py:28-30).
__host__ __device__ __forceinline__ int m2l_source_entry(const int32_t *__restrict__ ncoll, const int32_t *__restrict__ nent,
                                                const int32_t *__restrict__ nbot, const int32_t *__restrict__ ntop,
                                                int p, int d) {
    const int nb = ncoll[9 * (size_t)p + d];
    if (nb < 0) return -1;
    const int je = nent[nb];
    return (je >= 0 && ntop[nb] > nbot[nb]) ? je : -1;
}

// ------------------------------------------------------ host-side helpers
inline unsigned grid_for(int64_t n, int block, int cap = 1 << 20) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// tree.cu
void build_tree(kifmm_plan *P, const double *x, const double *y, int64_t n, int mem);
void export_tree(kifmm_plan *P, int64_t *nodes, int64_t *point_leaf);
void export_lists(kifmm_plan *P, int64_t *coll, int64_t *m2l, int64_t *n_m2l, int64_t *p2p, int64_t *n_p2p);
void tree_stats(kifmm_plan *P);
// operators.cu
void build_operators(kifmm_plan *P);
void init_log_table(int device);     // table of the Laplace P2M logarithm, once per device
void ensure_side(kifmm_plan *P);      // side stream and its events
void start_operators(kifmm_plan *P, bool fork_recorded = false);  // build_operators on the side stream
cudaStream_t device_side_stream(int device);  // one per device, created on first use
void join_operators(kifmm_plan *P);   // main stream waits for it
void ops_wait_now(kifmm_plan *P);     // issue a deferred join's stream wait (before any operator is read)
void ops_wait_circles(kifmm_plan *P); // ... for the check circles only (before the P2M)
void near_join(kifmm_plan *P);        // main stream waits for a near-field pass in flight, which is dropped
bool near_possible(kifmm_plan *P);    // passes_mixed.cu: whether the apply runs the near field on its own stream
void ensure_aux_streams(kifmm_plan *P); // passes_mixed.cu: the plan's near / far streams
// Runs what the scope enqueues on the plan's far stream (highest priority):
// forked from the plan's stream at construction, launches and allocations
// swapped there, joined back into the plan's stream at destruction.
struct HighPriorityFork {
    kifmm_plan *P;
    bool on;
    cudaStream_t main, g;
    HighPriorityFork(kifmm_plan *p, bool fork) : P(p), on(fork), main(p->stream), g(g_stream) {
        if (!on) return;
        KIFMM_CUDA(cudaEventRecord(P->far_fork, main));
        KIFMM_CUDA(cudaStreamWaitEvent(P->far_stream, P->far_fork, 0));
        P->stream = P->far_stream;
        g_stream = P->far_stream;
    }
    ~HighPriorityFork() {
        if (!on) return;
        cudaEventRecord(P->far_done, P->far_stream);
        P->stream = main;
        g_stream = g;
        cudaStreamWaitEvent(main, P->far_done, 0);
    }
    HighPriorityFork(const HighPriorityFork &) = delete;
    HighPriorityFork &operator=(const HighPriorityFork &) = delete;
};
// planned.cu
bool planned_ready(const kifmm_plan *P);
void build_plan_matrices(kifmm_plan *P);
// passes.cu
void run_upward_downward(kifmm_plan *P);
void run_eval_sources(kifmm_plan *P, int check_self);
void run_eval_targets(kifmm_plan *P, const double *tx, const double *ty, int64_t n, int check_self, double *pot);
void direct_sum_device(const kifmm_kernel &k, const double *x, const double *y, const double *tau, int64_t n,
                       const int64_t *tg, int64_t nt, double *out, cudaStream_t s);
void kernel_matrix_device(const kifmm_kernel &k, const double *sx, const double *sy, int64_t ns,
                          const double *tx, const double *ty, int64_t nt, double *out, cudaStream_t s);
void kernel_apply_device(const kifmm_kernel &k, const double *sx, const double *sy, int64_t ns,
                         const double *tx, const double *ty, int64_t nt, const double *tau, double *out,
                         cudaStream_t s);
// m2l_tc.cu
void build_tc_operators(kifmm_plan *P);
bool uses_tensor_m2l(const kifmm_plan *P);
// radix_sort.cu
void radix_sort_pairs(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, int bits,
                      kifmm_plan *P);
void radix_sort_keys(uint64_t *key, uint64_t *key_tmp, int64_t n, int bits, kifmm_plan *P);
void radix_sort_keys_shifts(uint64_t *key, uint64_t *key_tmp, int64_t n, const int *shifts, int npass,
                            kifmm_plan *P);
void radix_sort_pairs_bits(uint64_t *key, int32_t *val, uint64_t *key_tmp, int32_t *val_tmp, int64_t n, int lo_bit,
                           int bits, kifmm_plan *P);

}  // namespace kifmm
