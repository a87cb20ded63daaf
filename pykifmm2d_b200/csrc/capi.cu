// capi.cu -- the extern "C" entry points declared in include/kifmm2d.h.
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "kifmm_internal.cuh"
#include "passes.cuh"

namespace kifmm {

static thread_local std::string g_last_error;
std::atomic<long long> g_launch_count{0};
thread_local cudaStream_t g_stream = nullptr;

// Keep up to this many bytes of freed blocks cached in the device's default
// memory pool, so that plans created per point set reuse memory instead of
// returning it to the driver.
static const uint64_t kPoolKeepBytes = 8ull << 30;
static bool g_pool_ready[64] = {};
static void prepare_pool(int device) {
    if (device < 0 || device >= 64 || g_pool_ready[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = kPoolKeepBytes;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_pool_ready[device] = true;
}

PhaseScope::PhaseScope(kifmm_plan *p, int phase) : P(p), id(phase) {
    if (!P->profiling) return;
    l0 = g_launch_count.load();
    if (cudaEventCreate(&a) == cudaSuccess) cudaEventRecord(a, P->stream);
    else a = nullptr;
}

PhaseScope::~PhaseScope() {
    if (!a) return;
    cudaEvent_t b = nullptr;
    if (cudaEventCreate(&b) == cudaSuccess && cudaEventRecord(b, P->stream) == cudaSuccess) {
        P->pending.push_back(PendingPhase{id, a, b, g_launch_count.load() - l0});
    } else {
        cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
}

static void resolve_phases(kifmm_plan *P) {
    if (P->pending.empty()) return;
    KIFMM_CUDA(cudaStreamSynchronize(P->stream));
    if (P->near_stream) KIFMM_CUDA(cudaStreamSynchronize(P->near_stream));
    for (auto &ph : P->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ph.a, ph.b) == cudaSuccess) P->phase_ms[ph.id] += ms;
        P->phase_launches[ph.id] += ph.launches;
        cudaEventDestroy(ph.a);
        cudaEventDestroy(ph.b);
    }
    P->pending.clear();
}

// Pinned host blocks of HP_WORDS words, recycled across plans (a pinned
// allocation costs far more than a plan's other setup).
static std::mutex g_pin_mu;
static std::vector<unsigned long long *> g_pin_free;
unsigned long long *pinned_acquire() {
    unsigned long long *p = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pin_mu);
        if (!g_pin_free.empty()) {
            p = g_pin_free.back();
            g_pin_free.pop_back();
        }
    }
    if (!p) KIFMM_CUDA(cudaHostAlloc((void **)&p, HP_WORDS * sizeof(unsigned long long), cudaHostAllocPortable));
    for (int i = 0; i < HP_WORDS; i++) p[i] = 0;
    p[HP_INIT + 0] = p[HP_INIT + 2] = ~0ull;
    return p;
}
void pinned_release(unsigned long long *p) {
    std::lock_guard<std::mutex> lock(g_pin_mu);
    g_pin_free.push_back(p);
}

void ensure_dyn_smem(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> done;
    int dev = 0;
    KIFMM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = done[{dev, fn}];
    if (bytes <= cur) return;
    KIFMM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

cudaStream_t device_side_stream(int device) {
    static std::mutex mu;
    static cudaStream_t side[64] = {};
    KIFMM_REQUIRE(device >= 0 && device < 64, KIFMM_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!side[device]) KIFMM_CUDA(cudaStreamCreateWithFlags(&side[device], cudaStreamNonBlocking));
    return side[device];
}

// Build the tree on the plan's highest-priority stream (1) or on its own (0).
#ifndef KIFMM_TREE_FORK
#define KIFMM_TREE_FORK 1
#endif

// Pairs of (lowest-priority, highest-priority) streams for the plans' near
// field and far-field chain, kept per device and handed from a destroyed plan
// to the next one (creating two streams per plan costs more than a small
// apply's launches; stream-ordered frees on them stay valid across plans).
static std::mutex g_aux_mu;
static std::vector<std::pair<cudaStream_t, cudaStream_t>> g_aux_free[64];
void aux_streams_acquire(int device, cudaStream_t *near, cudaStream_t *far) {
    KIFMM_REQUIRE(device >= 0 && device < 64, KIFMM_ERR_ARG, "device index out of range");
    {
        std::lock_guard<std::mutex> lock(g_aux_mu);
        if (!g_aux_free[device].empty()) {
            *near = g_aux_free[device].back().first;
            *far = g_aux_free[device].back().second;
            g_aux_free[device].pop_back();
            return;
        }
    }
    int least = 0, greatest = 0;
    KIFMM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    KIFMM_CUDA(cudaStreamCreateWithPriority(near, cudaStreamNonBlocking, least));
    KIFMM_CUDA(cudaStreamCreateWithPriority(far, cudaStreamNonBlocking, greatest));
}
static void aux_streams_release(int device, cudaStream_t near, cudaStream_t far) {
    std::lock_guard<std::mutex> lock(g_aux_mu);
    g_aux_free[device].emplace_back(near, far);
}

// The plans' own streams (plans created without one), pooled the same way.
static std::vector<cudaStream_t> g_own_free[64];
static cudaStream_t own_stream_acquire(int device) {
    KIFMM_REQUIRE(device >= 0 && device < 64, KIFMM_ERR_ARG, "device index out of range");
    {
        std::lock_guard<std::mutex> lock(g_aux_mu);
        if (!g_own_free[device].empty()) {
            cudaStream_t s = g_own_free[device].back();
            g_own_free[device].pop_back();
            return s;
        }
    }
    cudaStream_t s = nullptr;
    KIFMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}
static void own_stream_release(int device, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(g_aux_mu);
    g_own_free[device].push_back(s);
}

void set_error(const std::string &msg) { g_last_error = msg; }

template <class F>
static int guarded(F &&f) {
    try {
        g_last_error.clear();
        f();
        return KIFMM_OK;
    } catch (const Fail &e) {
        return e.code;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return KIFMM_ERR_NOMEM;
    } catch (...) {
        set_error("unexpected C++ exception");
        return KIFMM_ERR_CUDA;
    }
}

static void use_device(kifmm_plan *P) {
    KIFMM_CUDA(cudaSetDevice(P->device));
    g_stream = P->stream;
}

static void copy_in(kifmm_plan *P, DBuf<double> &dst, const double *src, int64_t n, int mem) {
    KIFMM_REQUIRE(src || n == 0, KIFMM_ERR_ARG, "null input pointer");
    KIFMM_REQUIRE(mem == KIFMM_MEM_HOST || mem == KIFMM_MEM_DEVICE, KIFMM_ERR_ARG, "bad mem flag");
    dst.alloc(n);
    if (n)
        KIFMM_CUDA(cudaMemcpyAsync(dst.p, src, n * sizeof(double),
                                   mem == KIFMM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                   P->stream));
}

// Device-side failures reported through a flag (a tensor-core M2L wait that
// ran out of its poll budget); read after the stream has drained.
static void check_device_flags(kifmm_plan *P) {
    if (!P->scal.p || !P->hpin) return;
    unsigned long long *f = P->hpin + HP_FLAGS;
    KIFMM_CUDA(cudaMemcpyAsync(f, P->scal.p + KIFMM_SCAL_PASS_ERR, 2 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, P->stream));
    KIFMM_CUDA(cudaStreamSynchronize(P->stream));
    KIFMM_REQUIRE(f[0] == 0, KIFMM_ERR_CUDA, "M2M/L2L pass: a bulk-copy wait timed out");
    KIFMM_REQUIRE(f[1] == 0, KIFMM_ERR_CUDA, "tensor-core M2L: an MMA completion wait timed out");
}

static void copy_out(kifmm_plan *P, double *dst, const double *src, int64_t n, int mem) {
    KIFMM_REQUIRE(dst || n == 0, KIFMM_ERR_ARG, "null output pointer");
    if (n)
        KIFMM_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double),
                                   mem == KIFMM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                   P->stream));
    if (mem == KIFMM_MEM_HOST) {
        KIFMM_CUDA(cudaStreamSynchronize(P->stream));
        check_device_flags(P);
    }
}

static void check_kernel(const kifmm_kernel *k) {
    KIFMM_REQUIRE(k, KIFMM_ERR_ARG, "null kernel descriptor");
    KIFMM_REQUIRE(k->kind == KIFMM_KERNEL_LAPLACE || k->kind == KIFMM_KERNEL_MOD_HELMHOLTZ ||
                      k->kind == KIFMM_KERNEL_HELMHOLTZ,
                  KIFMM_ERR_ARG, "unknown kernel kind");
    KIFMM_REQUIRE(k->kind == KIFMM_KERNEL_LAPLACE || k->k > 0, KIFMM_ERR_ARG,
                  "(modified) Helmholtz needs k > 0");
}
// doubles per density / potential value of a kernel called outside a plan
static int64_t kernel_width(const kifmm_kernel *k) { return k->kind == KIFMM_KERNEL_HELMHOLTZ ? 2 : 1; }

// Stand-alone kernel-function calls (KF/KA/KAS) run on a temporary stream.
struct TempCtx {
    kifmm_plan P;
    explicit TempCtx(int device) {
        P.device = device;
        KIFMM_CUDA(cudaSetDevice(device));
        KIFMM_CUDA(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
        P.own_stream = true;
        g_stream = P.stream;
    }
    ~TempCtx() {
        if (P.stream) cudaStreamDestroy(P.stream);
    }
};

// serving batches: phases of the mixed apply (passes.cu, passes_mixed.cu)
// and the packed launches (m2l_tc.cu, passes_mixed.cu)
void apply_prologue(kifmm_plan *P);
void mixed_upward(kifmm_plan *P, const PassArgs &A);
void mixed_l2l(kifmm_plan *P, const PassArgs &A);
PassArgs mixed_leaf_args(kifmm_plan *P);
void launch_scatter_pot(kifmm_plan *P);
void launch_leaf_f_batch(int kind, const PassArgs *dargs, const int64_t *doff, int nplan, int64_t nleaf,
                         cudaStream_t s);
bool uses_tensor_m2l(const kifmm_plan *P);
int tc_form(const kifmm_plan *P);
size_t tc_args_bytes();
int64_t tc_prepare_batch(kifmm_plan *P, const PassArgs &A, void *args);
void launch_m2l_tc_batch(int form, const void *dargs, const int64_t *doff, int nplan, int64_t tiles,
                         cudaStream_t s);
// draws.cu
void launch_fill_normal(double *out, int64_t n, uint64_t seed, uint64_t index, cudaStream_t s);
void launch_fill_lanes(const void *dlanes, int nlanes, int64_t nmax, cudaStream_t s);
void launch_lane_sums(const void *dlanes, int nlanes, double *sums, cudaStream_t s);
size_t draw_lane_bytes();
void set_draw_lane(void *lanes, int r, double *out, int64_t n, uint64_t seed, uint64_t index);
void set_draw_seed(void *lanes, int r, uint64_t seed, uint64_t index);
constexpr uint64_t kDrawSkipSeed = ~0ull;

}  // namespace kifmm

using namespace kifmm;

// A packed apply of several plans, captured as one CUDA graph
// (kifmm_batch_capture).  The device tables hold the per-plan arguments of
// the two packed launches and the prefix sums of their work items.
struct kifmm_batch {
    std::vector<kifmm_plan *> plans;
    int device = 0;
    cudaStream_t stream = nullptr;      // the caller's stream
    std::vector<cudaStream_t> branch;   // one per plan
    std::vector<cudaEvent_t> ev;        // one per plan, then the fork event
    unsigned char *d_tc = nullptr;      // [nplan] M2L arguments
    int64_t *d_tc_off = nullptr;        // [nplan + 1] first tile of each plan
    PassArgs *d_leaf[2] = {};           // per kernel kind: leaf-pass arguments
    int64_t *d_leaf_off[2] = {};        // and the first leaf of each plan
    int64_t tiles = 0, leaves = 0;
    std::vector<unsigned char> h_draw;  // [nplan] density draws of the next launch (host copy)
    unsigned char *d_draw = nullptr;    // the same on the device, read by the graph's first kernel
    unsigned char *d_sumlane = nullptr; // [nplan] (pot_dev, n): the lanes summed by the last kernel
    double *d_sums = nullptr;           // [nplan] sums of the last launch
    double *h_sums = nullptr;           // pinned copy (kifmm_batch_synchronize)
    int64_t nmax = 0;
    cudaGraphExec_t graph = nullptr;
    ~kifmm_batch() {
        cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(d_draw);
        cudaFree(d_sumlane);
        cudaFree(d_sums);
        if (h_sums) cudaFreeHost(h_sums);
        for (auto s : branch) cudaStreamDestroy(s);
        for (auto e : ev) cudaEventDestroy(e);
        cudaFree(d_tc);
        cudaFree(d_tc_off);
        for (int k = 0; k < 2; k++) {
            cudaFree(d_leaf[k]);
            cudaFree(d_leaf_off[k]);
        }
    }
};

extern "C" {

void kifmm_default_options(kifmm_options *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->precision = KIFMM_PREC_FP64;
    o->m2l = KIFMM_M2L_AUTO;
}

int kifmm_plan_create(const kifmm_kernel *kernel, int32_t nequiv, int32_t ncutoff, const kifmm_options *opts,
                      kifmm_plan **plan_out) {
    return guarded([&] {
        KIFMM_REQUIRE(plan_out, KIFMM_ERR_ARG, "null plan_out");
        *plan_out = nullptr;
        check_kernel(kernel);
        KIFMM_REQUIRE(nequiv >= 4 && nequiv <= 64, KIFMM_ERR_ARG, "Nequiv must be in [4, 64]");
        const bool cplx = (opts && opts->iscomplex) || kernel->kind == KIFMM_KERNEL_HELMHOLTZ;
        if (cplx) {
            KIFMM_REQUIRE(nequiv <= 32, KIFMM_ERR_ARG, "Nequiv must be in [4, 32] for complex values");
            KIFMM_REQUIRE(!opts || opts->precision == KIFMM_PREC_FP64, KIFMM_ERR_UNSUPPORTED,
                          "complex values: only the FP64 precision form is built");
            KIFMM_REQUIRE(!opts || opts->e2c == KIFMM_E2C_DENSE, KIFMM_ERR_UNSUPPORTED,
                          "complex values: the circulant E2C solve is for real kernels");
            KIFMM_REQUIRE(!opts || !opts->planned, KIFMM_ERR_UNSUPPORTED,
                          "complex values: planned applies are for real values");
        }
        KIFMM_REQUIRE(ncutoff >= 1, KIFMM_ERR_ARG, "Ncutoff must be >= 1");
        kifmm_options o;
        kifmm_default_options(&o);
        if (opts) o = *opts;
        KIFMM_REQUIRE(o.precision == KIFMM_PREC_FP64 || o.precision == KIFMM_PREC_MIXED, KIFMM_ERR_ARG,
                      "unknown precision");
        KIFMM_REQUIRE(o.m2l >= KIFMM_M2L_AUTO && o.m2l <= KIFMM_M2L_INT8X4, KIFMM_ERR_ARG, "unknown M2L form");
        if (o.precision == KIFMM_PREC_MIXED && o.m2l == KIFMM_M2L_AUTO) o.m2l = KIFMM_M2L_INT8;
        KIFMM_REQUIRE(o.radii == 0 || o.radii == 1, KIFMM_ERR_ARG, "unknown radii preset");
        KIFMM_REQUIRE(o.e2c == KIFMM_E2C_DENSE || o.e2c == KIFMM_E2C_CIRCULANT, KIFMM_ERR_ARG,
                      "unknown E2C solve");
        KIFMM_REQUIRE(!(o.precision == KIFMM_PREC_MIXED && o.m2l == KIFMM_M2L_FP64), KIFMM_ERR_ARG,
                      "an FP64 M2L belongs to the FP64 precision form");
        kifmm_plan *P = new kifmm_plan();
        P->kern = *kernel;
        P->cplx = cplx;
        P->Qc = nequiv;
        P->Q = cplx ? 2 * nequiv : nequiv;  // complex: node state = [Re, Im] of the check potential
        o.iscomplex = cplx;
        P->ppl = ncutoff;
        P->opt = o;
        P->device = o.device;
        try {
            KIFMM_CUDA(cudaSetDevice(P->device));
            int sms = 0;
            KIFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->device));
            P->num_sms = sms > 0 ? sms : 148;
            prepare_pool(P->device);
            init_log_table(P->device);
            P->hpin = pinned_acquire();
            if (o.stream) {
                P->stream = (cudaStream_t)o.stream;
            } else {
                P->stream = own_stream_acquire(P->device);
                P->own_stream = true;
            }
        } catch (...) {
            delete P;
            throw;
        }
        *plan_out = P;
    });
}

static void drop_graph(kifmm_plan *P) {
    if (P->graph) cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
}

int kifmm_build_tree(kifmm_plan *P, const double *x, const double *y, int64_t n, int32_t mem) {
    return guarded([&] {
        if (P) drop_graph(P);
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(mem == KIFMM_MEM_HOST || mem == KIFMM_MEM_DEVICE, KIFMM_ERR_ARG, "bad mem flag");
        use_device(P);
        PhaseScope ph(P, KIFMM_PHASE_TREE);
        P->have_mats = false;
        P->applied = false;
        near_join(P);
        // the tree build's many small launches on the plan's highest-priority
        // stream, ahead of the operator build that it starts on the side stream
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        KIFMM_CUDA(cudaStreamIsCapturing(P->stream, &cap));
        const bool fork = KIFMM_TREE_FORK && cap == cudaStreamCaptureStatusNone;
        if (fork) ensure_aux_streams(P);
        HighPriorityFork hp(P, fork);
        build_tree(P, x, y, n, mem);
    });
}

int kifmm_precompute(kifmm_plan *P) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        use_device(P);
        PhaseScope ph(P, KIFMM_PHASE_PRECOMPUTE);
        KIFMM_REQUIRE(P->have_tree, KIFMM_ERR_STATE, "precompute: build_tree first");
        drop_graph(P);
        P->have_mats = false;
        P->applied = false;
        if (P->ops_pending) join_operators(P);  // started by build_tree
        else build_operators(P);
    });
}

int kifmm_build_expansions(kifmm_plan *P, const double *tau, int32_t mem) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(P->have_ops, KIFMM_ERR_STATE, "build_expansions: call precompute first");
        use_device(P);
        P->have_expansions = false;
        copy_in(P, P->tau, tau, P->cplx ? 2 * P->N : P->N, mem);
        run_upward_downward(P);
        P->have_expansions = true;
    });
}

int kifmm_evaluate_to_sources(kifmm_plan *P, double *pot, int32_t check_self, int32_t mem) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(P->have_expansions, KIFMM_ERR_STATE, "evaluate: call build_expansions first");
        KIFMM_REQUIRE(mem == KIFMM_MEM_HOST || mem == KIFMM_MEM_DEVICE, KIFMM_ERR_ARG, "bad mem flag");
        use_device(P);
        run_eval_sources(P, check_self != 0);
        P->applied = true;
        copy_out(P, pot, P->pot_out.p, P->cplx ? 2 * P->N : P->N, mem);
    });
}

int kifmm_evaluate_to_points(kifmm_plan *P, const double *x, const double *y, int64_t n, int32_t check_self,
                             double *pot, int32_t mem) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(P->have_expansions, KIFMM_ERR_STATE, "evaluate: call build_expansions first");
        KIFMM_REQUIRE(n >= 0, KIFMM_ERR_ARG, "negative target count");
        use_device(P);
        if (n == 0) return;
        copy_in(P, P->tx, x, n, mem);
        copy_in(P, P->ty, y, n, mem);
        const int64_t vw = P->cplx ? 2 : 1;
        P->tpot.alloc(n * vw);
        {
            PhaseScope ph(P, KIFMM_PHASE_TARGETS);
            run_eval_targets(P, P->tx.p, P->ty.p, n, check_self != 0, P->tpot.p);
        }
        copy_out(P, pot, P->tpot.p, n * vw, mem);
    });
}

int kifmm_synchronize(kifmm_plan *P) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        use_device(P);
        ops_wait_now(P);
        if (P->near_pending) KIFMM_CUDA(cudaStreamWaitEvent(P->stream, P->near_done, 0));  // kept pending
        KIFMM_CUDA(cudaStreamSynchronize(P->stream));
        check_device_flags(P);
    });
}

// One apply on device pointers, no host synchronisation: what the graph holds.
static void apply_device(kifmm_plan *P, const double *tau, double *pot, bool check_self) {
    const int64_t nv = P->cplx ? 2 * P->N : P->N;
    P->tau.alloc(nv);
    KIFMM_CUDA(cudaMemcpyAsync(P->tau.p, tau, nv * sizeof(double), cudaMemcpyDeviceToDevice, P->stream));
    run_upward_downward(P);
    run_eval_sources(P, check_self);
    KIFMM_CUDA(cudaMemcpyAsync(pot, P->pot_out.p, nv * sizeof(double), cudaMemcpyDeviceToDevice, P->stream));
    P->applied = true;
}

int kifmm_graph_capture(kifmm_plan *P, const double *tau, double *pot, int32_t check_self) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(tau && pot, KIFMM_ERR_ARG, "null device pointer");
        KIFMM_REQUIRE(P->have_ops, KIFMM_ERR_STATE, "graph capture: call precompute first");
        KIFMM_REQUIRE(P->stream && P->stream != cudaStreamLegacy && P->stream != cudaStreamPerThread,
                      KIFMM_ERR_ARG, "graph capture: the plan needs a created stream, not a default stream");
        use_device(P);
        drop_graph(P);
        const bool prof = P->profiling;
        P->profiling = false;  // no timer events inside the graph
        struct Restore {
            kifmm_plan *P;
            bool prof;
            ~Restore() { P->profiling = prof; }
        } restore{P, prof};
        apply_device(P, tau, pot, check_self != 0);  // allocates; sets kernel attributes
        P->have_expansions = true;
        KIFMM_CUDA(cudaStreamSynchronize(P->stream));
        check_device_flags(P);
        KIFMM_CUDA(cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t g = nullptr;
        try {
            apply_device(P, tau, pot, check_self != 0);
        } catch (...) {
            cudaStreamEndCapture(P->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        KIFMM_CUDA(cudaStreamEndCapture(P->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&P->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            P->graph = nullptr;
            KIFMM_CUDA(e);
        }
    });
}

int kifmm_graph_launch(kifmm_plan *P) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(P->graph, KIFMM_ERR_STATE, "graph launch: call kifmm_graph_capture first");
        use_device(P);
        KIFMM_CUDA(cudaGraphLaunch(P->graph, P->stream));
    });
}

int kifmm_get_tree_info(kifmm_plan *P, kifmm_tree_info *info) {
    return guarded([&] {
        KIFMM_REQUIRE(P && info, KIFMM_ERR_ARG, "null argument");
        KIFMM_REQUIRE(P->have_tree, KIFMM_ERR_STATE, "tree_info: no tree");
        use_device(P);
        tree_stats(P);
        memset(info, 0, sizeof(*info));
        info->n_points = P->N;
        info->levels = P->L;
        info->n_nodes = P->n_nodes;
        info->n_leaves = P->n_leaves;
        info->n_fake = P->n_fake;
        info->n_xlist = P->n_xlist;
        info->n_outside = P->n_outside;
        info->root_min = P->root_min;
        info->root_max = P->root_max;
        info->n_p2p_pairs = P->n_p2p_pairs;
        info->n_p2m_points = P->n_p2m_points;
        info->n_m2l_pairs = P->n_m2l_pairs;
        info->n_m2l_groups = P->n_m2l_groups;
        for (int l = 0; l < P->L && l < KIFMM_MAX_LEVELS; l++) info->nodes_per_level[l] = P->lv[l].n;
        info->planned_bytes = P->have_mats ? (int64_t)P->pm_bytes : 0;
    });
}

int kifmm_export_tree(kifmm_plan *P, int64_t *nodes, int64_t *point_leaf) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        use_device(P);
        export_tree(P, nodes, point_leaf);
    });
}

int kifmm_export_lists(kifmm_plan *P, int64_t *colleagues, int64_t *m2l, int64_t *n_m2l, int64_t *p2p,
                       int64_t *n_p2p) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        KIFMM_REQUIRE(!m2l || n_m2l, KIFMM_ERR_ARG, "export_lists: m2l needs its capacity in *n_m2l");
        KIFMM_REQUIRE(!p2p || n_p2p, KIFMM_ERR_ARG, "export_lists: p2p needs its capacity in *n_p2p");
        use_device(P);
        export_lists(P, colleagues, m2l, n_m2l, p2p, n_p2p);
    });
}

int kifmm_plan_destroy(kifmm_plan *P) {
    return guarded([&] {
        if (!P) return;
        cudaSetDevice(P->device);
        g_stream = P->stream;
        drop_graph(P);
        for (auto &ph : P->pending) { cudaEventDestroy(ph.a); cudaEventDestroy(ph.b); }
        P->pending.clear();
        cudaStream_t s = P->stream, side = P->side;
        cudaEvent_t e0 = P->ops_fork, e1 = P->ops_done, e2 = P->tree_ev, e3 = P->ops_circ;
        cudaStream_t ns = P->near_stream, fs = P->far_stream;
        cudaEvent_t n0 = P->near_fork, n1 = P->near_done, f0 = P->far_fork, f1 = P->far_done;
        const int dev = P->device;
        if (ns) cudaStreamSynchronize(ns);  // a near-field pass still reading the plan's buffers
        bool own = P->own_stream;
        unsigned long long *hp = P->hpin;
        delete P;  // buffers are freed stream-ordered on s and on the side stream
        if (s) cudaStreamSynchronize(s);
        if (hp) pinned_release(hp);
        if (side) {  // the device's shared side stream stays
            cudaStreamSynchronize(side);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaEventDestroy(e2);
            cudaEventDestroy(e3);
        }
        if (ns) {  // buffers allocated on the far stream were freed on it by the plan's destructor
            cudaStreamSynchronize(fs);
            cudaEventDestroy(n0);
            cudaEventDestroy(n1);
            cudaEventDestroy(f0);
            cudaEventDestroy(f1);
            aux_streams_release(dev, ns, fs);
        }
        if (own && s) own_stream_release(dev, s);  // synchronised above
    });
}

const char *kifmm_last_error(void) { return g_last_error.c_str(); }

int kifmm_direct_sum(const kifmm_kernel *kernel, const double *x, const double *y, const double *tau, int64_t n,
                     const int64_t *targets, int64_t nt, double *out, int32_t mem, int32_t device) {
    return guarded([&] {
        check_kernel(kernel);
        KIFMM_REQUIRE(n > 0 && nt >= 0, KIFMM_ERR_ARG, "bad sizes");
        TempCtx C(device);
        kifmm_plan *P = &C.P;
        DBuf<double> dx, dy, dt, dout;
        DBuf<int64_t> dtg;
        const double *px = x, *py = y, *pt = tau;
        const int64_t *ptg = targets;
        double *po = out;
        if (mem == KIFMM_MEM_HOST) {
            KIFMM_REQUIRE(targets || nt == 0, KIFMM_ERR_ARG, "null targets");
            for (int64_t a = 0; a < nt; a++)
                KIFMM_REQUIRE(targets[a] >= 0 && targets[a] < n, KIFMM_ERR_ARG, "target index out of range");
            const int64_t vw = kernel_width(kernel);
            copy_in(P, dx, x, n, mem); copy_in(P, dy, y, n, mem); copy_in(P, dt, tau, n * vw, mem);
            dtg.alloc(nt);
            KIFMM_CUDA(cudaMemcpyAsync(dtg.p, targets, nt * sizeof(int64_t), cudaMemcpyHostToDevice, P->stream));
            dout.alloc(nt * vw);
            px = dx.p; py = dy.p; pt = dt.p; ptg = dtg.p; po = dout.p;
        }
        direct_sum_device(*kernel, px, py, pt, n, ptg, nt, po, P->stream);
        if (mem == KIFMM_MEM_HOST) copy_out(P, out, dout.p, nt * kernel_width(kernel), mem);
        KIFMM_CUDA(cudaStreamSynchronize(P->stream));
    });
}

int kifmm_kernel_matrix(const kifmm_kernel *kernel, const double *sx, const double *sy, int64_t ns, const double *tx,
                        const double *ty, int64_t nt, double *out, int32_t mem, int32_t device) {
    return guarded([&] {
        check_kernel(kernel);
        KIFMM_REQUIRE(ns >= 0 && nt >= 0, KIFMM_ERR_ARG, "bad sizes");
        TempCtx C(device);
        kifmm_plan *P = &C.P;
        DBuf<double> a, b, c, d, o;
        const double *psx = sx, *psy = sy, *ptx = tx, *pty = ty;
        double *po = out;
        if (mem == KIFMM_MEM_HOST) {
            copy_in(P, a, sx, ns, mem); copy_in(P, b, sy, ns, mem); copy_in(P, c, tx, nt, mem); copy_in(P, d, ty, nt, mem);
            o.alloc(ns * nt * kernel_width(kernel));
            psx = a.p; psy = b.p; ptx = c.p; pty = d.p; po = o.p;
        }
        kernel_matrix_device(*kernel, psx, psy, ns, ptx, pty, nt, po, P->stream);
        if (mem == KIFMM_MEM_HOST) copy_out(P, out, o.p, ns * nt * kernel_width(kernel), mem);
        KIFMM_CUDA(cudaStreamSynchronize(P->stream));
    });
}

int kifmm_kernel_apply(const kifmm_kernel *kernel, const double *sx, const double *sy, int64_t ns, const double *tx,
                       const double *ty, int64_t nt, const double *tau, double *out, int32_t mem, int32_t device) {
    return guarded([&] {
        check_kernel(kernel);
        KIFMM_REQUIRE(ns >= 0 && nt >= 0, KIFMM_ERR_ARG, "bad sizes");
        TempCtx C(device);
        kifmm_plan *P = &C.P;
        DBuf<double> a, b, c, d, t, o;
        const double *psx = sx, *psy = sy, *ptx = tx, *pty = ty, *pt = tau;
        double *po = out;
        if (mem == KIFMM_MEM_HOST) {
            copy_in(P, a, sx, ns, mem); copy_in(P, b, sy, ns, mem); copy_in(P, c, tx, nt, mem);
            copy_in(P, d, ty, nt, mem); copy_in(P, t, tau, ns * kernel_width(kernel), mem);
            o.alloc(nt * kernel_width(kernel));
            psx = a.p; psy = b.p; ptx = c.p; pty = d.p; pt = t.p; po = o.p;
        }
        kernel_apply_device(*kernel, psx, psy, ns, ptx, pty, nt, pt, po, P->stream);
        if (mem == KIFMM_MEM_HOST) copy_out(P, out, o.p, nt * kernel_width(kernel), mem);
        KIFMM_CUDA(cudaStreamSynchronize(P->stream));
    });
}

int kifmm_set_profiling(kifmm_plan *P, int32_t on) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        use_device(P);
        resolve_phases(P);
        P->profiling = on != 0;
    });
}

int kifmm_get_phase_times(kifmm_plan *P, double *ms, int64_t *launches, int32_t reset) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        use_device(P);
        resolve_phases(P);
        for (int i = 0; i < KIFMM_PHASE_COUNT; i++) {
            if (ms) ms[i] = P->phase_ms[i];
            if (launches) launches[i] = P->phase_launches[i];
            if (reset) { P->phase_ms[i] = 0; P->phase_launches[i] = 0; }
        }
    });
}

int kifmm_set_wait_limit(kifmm_plan *P, int64_t polls) {
    return guarded([&] {
        KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "null plan");
        drop_graph(P);  // a captured graph holds the old budget
        P->wait_limit = polls >= 0 ? (long long)polls : -1;
    });
}

static void check_batch_plan(kifmm_plan *P, int device, int form) {
    KIFMM_REQUIRE(P, KIFMM_ERR_ARG, "batch: null plan");
    KIFMM_REQUIRE(P->have_ops, KIFMM_ERR_STATE, "batch: every plan needs precompute first");
    KIFMM_REQUIRE(P->device == device, KIFMM_ERR_ARG, "batch: all plans must be on one device");
    KIFMM_REQUIRE(uses_tensor_m2l(P) && !P->opt.near_fp64 && !P->opt.planned && !P->cplx, KIFMM_ERR_ARG,
                  "batch: plans must use the mixed form with a tensor-core M2L (no near_fp64, planned or "
                  "complex option)");
    KIFMM_REQUIRE(tc_form(P) == form, KIFMM_ERR_ARG, "batch: all plans must use one M2L form");
    KIFMM_REQUIRE(P->kern.kind == KIFMM_KERNEL_LAPLACE || P->kern.kind == KIFMM_KERNEL_MOD_HELMHOLTZ,
                  KIFMM_ERR_ARG, "batch: Laplace or modified-Helmholtz plans only");
}

// Every plan's first phase (densities in, P2M, M2M, M2L slices) in its branch,
// the packed M2L, the L2L and leaf arguments in the branches, the packed leaf
// passes, then the scatters: fork and join through events, so that the capture
// holds the branches as parallel paths of one graph.
static void batch_record(kifmm_batch *B, const double *const *tau, double *const *pot,
                         std::vector<unsigned char> &htc, std::vector<int64_t> &htoff,
                         std::vector<PassArgs> (&hleaf)[2], std::vector<int64_t> (&hloff)[2]) {
    const int n = (int)B->plans.size();
    cudaEvent_t fork = B->ev[n];
    const size_t tcb = tc_args_bytes();
    auto fork_all = [&] {
        KIFMM_CUDA(cudaEventRecord(fork, B->stream));
        for (int r = 0; r < n; r++) KIFMM_CUDA(cudaStreamWaitEvent(B->branch[r], fork, 0));
    };
    auto join_all = [&] {
        for (int r = 0; r < n; r++) {
            KIFMM_CUDA(cudaEventRecord(B->ev[r], B->branch[r]));
            KIFMM_CUDA(cudaStreamWaitEvent(B->stream, B->ev[r], 0));
        }
    };
    launch_fill_lanes(B->d_draw, n, B->nmax, B->stream);  // lanes whose density the batch draws
    fork_all();
    htoff.assign(1, 0);
    for (int r = 0; r < n; r++) {
        kifmm_plan *P = B->plans[r];
        KIFMM_CUDA(cudaMemcpyAsync(P->tau.p, tau[r], P->N * sizeof(double), cudaMemcpyDeviceToDevice, P->stream));
        apply_prologue(P);
        int64_t t = 0;
        if (P->L >= 3) {
            PassArgs A = make_pass_args(P);
            mixed_upward(P, A);
            t = tc_prepare_batch(P, A, htc.data() + (size_t)r * tcb);
        }
        htoff.push_back(htoff.back() + t);
    }
    join_all();
    B->tiles = htoff.back();
    if (B->tiles) launch_m2l_tc_batch(tc_form(B->plans[0]), B->d_tc, B->d_tc_off, n, B->tiles, B->stream);
    fork_all();
    for (int k = 0; k < 2; k++) hloff[k].assign(1, 0), hleaf[k].clear();
    for (int r = 0; r < n; r++) {
        kifmm_plan *P = B->plans[r];
        if (P->L >= 3) mixed_l2l(P, make_pass_args(P));
        if (!P->n_leaf_list) continue;
        const int k = P->kern.kind == KIFMM_KERNEL_LAPLACE ? 0 : 1;
        hleaf[k].push_back(mixed_leaf_args(P));
        hloff[k].push_back(hloff[k].back() + P->n_leaf_list);
    }
    join_all();
    B->leaves = 0;
    for (int k = 0; k < 2; k++) {
        const int64_t nl = hloff[k].back();
        B->leaves += nl;
        if (nl)
            launch_leaf_f_batch(k == 0 ? KIFMM_KERNEL_LAPLACE : KIFMM_KERNEL_MOD_HELMHOLTZ, B->d_leaf[k],
                                B->d_leaf_off[k], (int)hleaf[k].size(), nl, B->stream);
    }
    fork_all();
    for (int r = 0; r < n; r++) {
        kifmm_plan *P = B->plans[r];
        launch_scatter_pot(P);
        KIFMM_CUDA(cudaMemcpyAsync(pot[r], P->pot_out.p, P->N * sizeof(double), cudaMemcpyDeviceToDevice,
                                   P->stream));
    }
    join_all();
    launch_lane_sums(B->d_sumlane, n, B->d_sums, B->stream);
}

int kifmm_batch_capture(kifmm_plan *const *plans, int32_t nplan, const double *const *tau, double *const *pot,
                        int32_t check_self, void *stream, kifmm_batch **batch_out) {
    return guarded([&] {
        KIFMM_REQUIRE(batch_out, KIFMM_ERR_ARG, "null output pointer");
        *batch_out = nullptr;
        KIFMM_REQUIRE(plans && tau && pot && nplan > 0 && nplan <= 4096, KIFMM_ERR_ARG,
                      "batch: bad plan list");
        cudaStream_t cs = (cudaStream_t)stream;
        KIFMM_REQUIRE(cs && cs != cudaStreamLegacy && cs != cudaStreamPerThread, KIFMM_ERR_ARG,
                      "batch: needs a created stream, not a default stream");
        KIFMM_REQUIRE(plans[0], KIFMM_ERR_ARG, "batch: null plan");
        const int device = plans[0]->device, form = tc_form(plans[0]);
        for (int r = 0; r < nplan; r++) {
            check_batch_plan(plans[r], device, form);
            KIFMM_REQUIRE(tau[r] && pot[r], KIFMM_ERR_ARG, "batch: null device pointer");
            for (int q = 0; q < r; q++) KIFMM_REQUIRE(plans[q] != plans[r], KIFMM_ERR_ARG, "batch: repeated plan");
        }
        KIFMM_CUDA(cudaSetDevice(device));
        std::unique_ptr<kifmm_batch> B(new kifmm_batch);
        B->device = device;
        B->stream = cs;
        B->plans.assign(plans, plans + nplan);
        for (int r = 0; r <= nplan; r++) {
            cudaEvent_t e;
            KIFMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            B->ev.push_back(e);
        }
        for (int r = 0; r < nplan; r++) {
            cudaStream_t st;
            KIFMM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            B->branch.push_back(st);
        }
        const size_t tcb = tc_args_bytes();
        KIFMM_CUDA(cudaMalloc(&B->d_tc, tcb * nplan));
        KIFMM_CUDA(cudaMalloc(&B->d_tc_off, sizeof(int64_t) * (nplan + 1)));
        for (int k = 0; k < 2; k++) {
            KIFMM_CUDA(cudaMalloc(&B->d_leaf[k], sizeof(PassArgs) * nplan));
            KIFMM_CUDA(cudaMalloc(&B->d_leaf_off[k], sizeof(int64_t) * (nplan + 1)));
        }
        const size_t dlb = draw_lane_bytes();
        B->h_draw.assign(dlb * nplan, 0);
        std::vector<unsigned char> hsum(dlb * nplan, 0);
        for (int r = 0; r < nplan; r++) {
            set_draw_lane(B->h_draw.data(), r, const_cast<double *>(tau[r]), plans[r]->N, kDrawSkipSeed, 0);
            set_draw_lane(hsum.data(), r, pot[r], plans[r]->N, kDrawSkipSeed, 0);
            B->nmax = std::max<int64_t>(B->nmax, plans[r]->N);
        }
        KIFMM_CUDA(cudaMalloc(&B->d_draw, dlb * nplan));
        KIFMM_CUDA(cudaMalloc(&B->d_sumlane, dlb * nplan));
        KIFMM_CUDA(cudaMalloc(&B->d_sums, sizeof(double) * nplan));
        KIFMM_CUDA(cudaMallocHost(&B->h_sums, sizeof(double) * nplan));
        KIFMM_CUDA(cudaMemcpy(B->d_draw, B->h_draw.data(), dlb * nplan, cudaMemcpyHostToDevice));
        KIFMM_CUDA(cudaMemcpy(B->d_sumlane, hsum.data(), dlb * nplan, cudaMemcpyHostToDevice));
        // a plan without an apply since its tree and operators were built runs
        // one on its own stream after the caller's work: that allocates every
        // apply buffer (stream-ordered on the plan's stream)
        KIFMM_CUDA(cudaEventRecord(B->ev[nplan], cs));
        for (int r = 0; r < nplan; r++) {
            kifmm_plan *P = plans[r];
            use_device(P);
            if (P->applied) continue;
            drop_graph(P);
            KIFMM_CUDA(cudaStreamWaitEvent(P->stream, B->ev[nplan], 0));
            const bool prof = P->profiling;
            P->profiling = false;
            apply_device(P, tau[r], pot[r], check_self != 0);
            P->profiling = prof;
            P->have_expansions = true;
            KIFMM_CUDA(cudaEventRecord(B->ev[r], P->stream));
            KIFMM_CUDA(cudaStreamWaitEvent(cs, B->ev[r], 0));
        }
        KIFMM_CUDA(cudaStreamSynchronize(cs));
        for (int r = 0; r < nplan; r++) {
            use_device(plans[r]);
            KIFMM_CUDA(cudaStreamSynchronize(plans[r]->stream));
            check_device_flags(plans[r]);
        }
        KIFMM_CUDA(cudaSetDevice(device));
        // capture with each plan's work ordered on its branch stream
        std::vector<cudaStream_t> own(nplan);
        std::vector<char> prof(nplan);
        for (int r = 0; r < nplan; r++) {
            own[r] = plans[r]->stream;
            prof[r] = plans[r]->profiling;
            plans[r]->stream = B->branch[r];
            plans[r]->profiling = false;
        }
        struct Restore {
            kifmm_plan *const *plans;
            const std::vector<cudaStream_t> &own;
            const std::vector<char> &prof;
            ~Restore() {
                for (size_t r = 0; r < own.size(); r++) {
                    plans[r]->stream = own[r];
                    plans[r]->profiling = prof[r];
                }
            }
        } restore{plans, own, prof};
        g_stream = own[0];  // no allocation is expected: the apply above made every buffer
        std::vector<unsigned char> htc(tcb * nplan, 0);
        std::vector<int64_t> htoff;
        std::vector<PassArgs> hleaf[2];
        std::vector<int64_t> hloff[2];
        // A call made by another host thread meanwhile that synchronises
        // implicitly with every stream (some allocations do) invalidates a
        // capture in progress; the capture is then made again.
        cudaGraph_t g = nullptr;
        for (int attempt = 0;; attempt++) {
            KIFMM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            bool failed = false;
            try {
                batch_record(B.get(), tau, pot, htc, htoff, hleaf, hloff);
            } catch (...) {
                failed = true;
                if (attempt >= 3) {
                    cudaStreamEndCapture(cs, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
            }
            const cudaError_t ee = cudaStreamEndCapture(cs, &g);
            if (!failed && ee == cudaSuccess) break;
            if (g) cudaGraphDestroy(g);
            g = nullptr;
            if (attempt >= 3) KIFMM_CUDA(ee != cudaSuccess ? ee : cudaErrorStreamCaptureInvalidated);
            cudaGetLastError();
        }
        cudaError_t e = cudaGraphInstantiate(&B->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            B->graph = nullptr;
            KIFMM_CUDA(e);
        }
        // the tables the packed kernels read, in place before the first launch
        KIFMM_CUDA(cudaMemcpy(B->d_tc, htc.data(), htc.size(), cudaMemcpyHostToDevice));
        KIFMM_CUDA(cudaMemcpy(B->d_tc_off, htoff.data(), htoff.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
        for (int k = 0; k < 2; k++) {
            if (!hleaf[k].empty())
                KIFMM_CUDA(cudaMemcpy(B->d_leaf[k], hleaf[k].data(), hleaf[k].size() * sizeof(PassArgs),
                                      cudaMemcpyHostToDevice));
            KIFMM_CUDA(cudaMemcpy(B->d_leaf_off[k], hloff[k].data(), hloff[k].size() * sizeof(int64_t),
                                  cudaMemcpyHostToDevice));
        }
        *batch_out = B.release();
    });
}

int kifmm_batch_launch(kifmm_batch *B) {
    return guarded([&] {
        KIFMM_REQUIRE(B && B->graph, KIFMM_ERR_ARG, "batch launch: no captured batch");
        KIFMM_CUDA(cudaSetDevice(B->device));
        KIFMM_CUDA(cudaGraphLaunch(B->graph, B->stream));
    });
}

int kifmm_batch_set_draws(kifmm_batch *B, const uint64_t *seed, const uint64_t *index) {
    return guarded([&] {
        KIFMM_REQUIRE(B && seed && index, KIFMM_ERR_ARG, "null argument");
        KIFMM_CUDA(cudaSetDevice(B->device));
        const int n = (int)B->plans.size();
        for (int r = 0; r < n; r++)
            set_draw_seed(B->h_draw.data(), r, seed[r], index[r]);
        // from pageable memory: the call returns once h_draw has been read
        KIFMM_CUDA(cudaMemcpyAsync(B->d_draw, B->h_draw.data(), B->h_draw.size(), cudaMemcpyHostToDevice,
                                   B->stream));
    });
}

int kifmm_batch_synchronize(kifmm_batch *B) {
    return guarded([&] {
        KIFMM_REQUIRE(B, KIFMM_ERR_ARG, "null batch");
        KIFMM_CUDA(cudaSetDevice(B->device));
        // every plan's error flags and the lane sums in one drain of the stream
        for (auto *P : B->plans)
            if (P->scal.p && P->hpin)
                KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_FLAGS, P->scal.p + KIFMM_SCAL_PASS_ERR,
                                           2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, B->stream));
        KIFMM_CUDA(cudaMemcpyAsync(B->h_sums, B->d_sums, sizeof(double) * B->plans.size(), cudaMemcpyDeviceToHost,
                                   B->stream));
        KIFMM_CUDA(cudaStreamSynchronize(B->stream));
        for (auto *P : B->plans) {
            if (!P->scal.p || !P->hpin) continue;
            const unsigned long long *f = P->hpin + HP_FLAGS;
            KIFMM_REQUIRE(f[0] == 0, KIFMM_ERR_CUDA, "M2M/L2L pass: a bulk-copy wait timed out");
            KIFMM_REQUIRE(f[1] == 0, KIFMM_ERR_CUDA, "tensor-core M2L: an MMA completion wait timed out");
        }
    });
}

int kifmm_batch_sums(kifmm_batch *B, double *sums) {
    return guarded([&] {
        KIFMM_REQUIRE(B && sums, KIFMM_ERR_ARG, "null argument");
        memcpy(sums, B->h_sums, sizeof(double) * B->plans.size());
    });
}

int kifmm_fill_normal(double *dev, int64_t n, uint64_t seed, uint64_t index, void *stream) {
    return guarded([&] {
        KIFMM_REQUIRE(n >= 0 && (dev || n == 0), KIFMM_ERR_ARG, "fill_normal: bad buffer");
        KIFMM_REQUIRE(seed != kDrawSkipSeed, KIFMM_ERR_ARG, "fill_normal: seed 2^64-1 is reserved");
        launch_fill_normal(dev, n, seed, index, (cudaStream_t)stream);
    });
}

int kifmm_batch_info(kifmm_batch *B, int64_t *m2l_tiles, int64_t *leaves) {
    return guarded([&] {
        KIFMM_REQUIRE(B, KIFMM_ERR_ARG, "null batch");
        if (m2l_tiles) *m2l_tiles = B->tiles;
        if (leaves) *leaves = B->leaves;
    });
}

int kifmm_batch_destroy(kifmm_batch *B) {
    return guarded([&] { delete B; });
}

int kifmm_stream_create(int32_t device, void **stream) {
    return guarded([&] {
        KIFMM_REQUIRE(stream, KIFMM_ERR_ARG, "null output pointer");
        KIFMM_REQUIRE(device >= 0 && device < 64, KIFMM_ERR_ARG, "device index out of range");
        KIFMM_CUDA(cudaSetDevice(device));
        cudaStream_t s = nullptr;
        KIFMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        *stream = (void *)s;
    });
}

int kifmm_stream_destroy(void *stream) {
    return guarded([&] {
        if (stream) KIFMM_CUDA(cudaStreamDestroy((cudaStream_t)stream));
    });
}

int64_t kifmm_launch_count(void) { return g_launch_count.load(); }

int kifmm_version(void) { return 100; }

}  // extern "C"
