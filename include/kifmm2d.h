/*
 * kifmm2d.h -- C ABI of the B200-native 2D kernel-independent FMM.
 *
 * The library (pykifmm2d_b200/libkifmm2d.so) replaces the hot path behind the
 * reference's Python class `FMM` (dbstein/pykifmm2d, pykifmm2d/class_fmm.py)
 * with hand-written sm_100a CUDA kernels.  Each entry point below names the
 * reference interface it replaces.  The Python layer pykifmm2d_b200 binds
 * these symbols with ctypes; other hosts can bind them the same way.
 *
 * Conventions
 *   - Every call returns a kifmm_status; nothing aborts or traps.  The text of
 *     the last error of the calling thread is kifmm_last_error().
 *   - `mem` says where a caller buffer lives: KIFMM_MEM_HOST (ordinary or
 *     pinned host memory; the call returns once the data is consumed or
 *     written) or KIFMM_MEM_DEVICE (device pointers on the plan's device;
 *     work is ordered on the plan's stream and the call may return before
 *     it finishes -- use kifmm_synchronize or the stream).
 *   - A plan owns its device memory.  The caller owns its input and output
 *     buffers.  One plan is used from one host thread at a time.
 */
#ifndef KIFMM2D_H
#define KIFMM2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    KIFMM_OK = 0,
    KIFMM_ERR_ARG = 1,        /* invalid argument (null pointer, bad size, NaN input, ...) */
    KIFMM_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    KIFMM_ERR_NOMEM = 3,      /* device allocation failed */
    KIFMM_ERR_DEPTH = 4,      /* tree would need more than KIFMM_MAX_LEVELS levels */
    KIFMM_ERR_STATE = 5,      /* call out of order (e.g. apply before build_tree) */
    KIFMM_ERR_RANGE = 6,      /* coordinates out of the exactly representable range */
    KIFMM_ERR_UNSUPPORTED = 7 /* option not supported by this build */
} kifmm_status;

enum { KIFMM_MEM_HOST = 0, KIFMM_MEM_DEVICE = 1 };

/* Opaque plan: tree, operators and workspaces of one FMM object. */
typedef struct kifmm_plan kifmm_plan;

/* Kernel plug-ins.  The reference takes a numba scalar function
 * Kernel_Eval(sx, sy, tx, ty) (class_fmm.py:55, :115); the ones it ships and
 * benchmarks are the Laplace log kernel (examples/laplace2.py:31-36), the
 * modified Helmholtz kernel K0(k r)/(2 pi) (examples/modified_helmholtz.py:38-43)
 * and, with FMM(..., iscomplex=True) (class_fmm.py:174), the Helmholtz kernel
 * (i/4) H0^(1)(k r) (examples/hankel.py:37-39).
 * Complex kernel: every density, potential and kernel value the ABI passes is
 * complex, stored as interleaved (real, imaginary) doubles (C99 double
 * complex / numpy complex128 layout), so a buffer of n values holds 2n
 * doubles; the plan needs KIFMM_PREC_FP64 and Nequiv <= 32. */
enum { KIFMM_KERNEL_LAPLACE = 0, KIFMM_KERNEL_MOD_HELMHOLTZ = 1, KIFMM_KERNEL_HELMHOLTZ = 2 };
typedef struct kifmm_kernel {
    int32_t kind;     /* KIFMM_KERNEL_* */
    int32_t reserved;
    double k;         /* wavenumber of the (modified) Helmholtz kernels (unused for Laplace) */
} kifmm_kernel;

/* Arithmetic of the evaluation passes. */
enum {
    KIFMM_PREC_FP64 = 0,  /* every pass in FP64 ("plain") */
    KIFMM_PREC_MIXED = 1  /* FP32 near field and P2M/L2P, compensated M2L */
};
/* M2L form used with KIFMM_PREC_MIXED. */
enum {
    KIFMM_M2L_AUTO = 0,       /* = KIFMM_M2L_INT8 */
    KIFMM_M2L_FP32 = 1,       /* FP32 FFMA tiles on the CUDA cores */
    KIFMM_M2L_BF16X3 = 2,     /* tcgen05 kind::f16, bf16 hi/lo, 3 products, FP32 accumulate */
    KIFMM_M2L_FP16X3 = 3,     /* tcgen05 kind::f16, fp16 hi/lo with scaling, 3 products */
    KIFMM_M2L_FP64 = 4,       /* FP64 tiles (the KIFMM_PREC_FP64 form) */
    KIFMM_M2L_INT8 = 5,       /* tcgen05 kind::i8: operator and vectors as five signed 7-bit
                                 slices, exact int32 accumulation, FP64 reconstruction */
    KIFMM_M2L_INT8X4 = 6      /* the same with four slices (10 slice products, ~2^-28 of the
                                 row and column scales instead of ~2^-35), 128 targets per tile */
};

typedef struct kifmm_options {
    int32_t precision;  /* KIFMM_PREC_* (default FP64) */
    int32_t m2l;        /* KIFMM_M2L_* (default AUTO) */
    int32_t fix_bbox;   /* 0 (default): the reference's root box
                           [floor(min(xmin,ymin)), ceil(max(xmax,ymin))] (tree.py:475-484);
                           1: use ymax, so every point lies inside the root box */
    int32_t radii;      /* 0 (default): the reference's circles r1=(sqrt2+0.01)w/2,
                           r2=(4-sqrt2-0.02)w/2 (class_fmm.py:35-45); 1: 1.5 and 2.5 half-widths */
    int32_t device;     /* CUDA device ordinal */
    int32_t near_fp64;  /* with KIFMM_PREC_MIXED: 1 keeps P2M, L2P and P2P in FP64 (only M2L
                           takes the mixed form); 0 (default): FP32 near field */
    void *stream;       /* cudaStream_t to order work on (cudaStreamLegacy, i.e. 0x1, for the
                           legacy default stream); NULL: the plan creates its own stream */
    int32_t e2c;        /* how the check-to-equivalent inverse is formed: KIFMM_E2C_* */
    int32_t iscomplex;  /* FMM(..., iscomplex=True) (class_fmm.py:174): 1 makes densities and
                           potentials complex (interleaved doubles) for any kernel; the
                           Helmholtz kernel sets it by itself.  0 (default): real values */
    int32_t planned;    /* the reference's planned FMM (fmm_planner / planned_fmm, fmm.py:530-814):
                           1 keeps the P2M, L2P and near-field kernel values of the tree in device
                           memory (built by the first apply after build_tree / precompute; about
                           8 B per near-field pair, 4 B in the mixed form, plus 16 Q B per point)
                           and applies them as matrices; evaluations at the sources with
                           check_self use them.  Real values only.  0 (default): on the fly */
    int32_t reserved;
} kifmm_options;

/* Check-to-equivalent solve.  The reference LU-factors the Q x Q E2C matrix
 * per level (class_fmm.py:213-217); its FFT variant diagonalises the same,
 * circulant, matrix by the DFT of its first row (svd_fmm.py:239-242,
 * :281-290): Q kernel evaluations and O(Q^2) work per level instead of Q^2
 * evaluations and an O(Q^3) factorisation. */
enum {
    KIFMM_E2C_DENSE = 0,     /* default: Gauss-Jordan inverse of the dense E2C (partial pivoting) */
    KIFMM_E2C_CIRCULANT = 1  /* inverse from the DFT eigenvalues of the circulant E2C */
};

#define KIFMM_MAX_LEVELS 30

typedef struct kifmm_tree_info {
    int64_t n_points;
    int32_t levels;          /* number of levels (reference Tree.levels) */
    int32_t reserved;
    int64_t n_nodes;         /* all nodes, fake leaves included */
    int64_t n_leaves;        /* real leaves (reference Level.leaf summed) */
    int64_t n_fake;          /* fake leaves made by X-list splits */
    int64_t n_xlist;         /* X-list leaves */
    int64_t n_outside;       /* points outside the root box (reference bbox quirk) */
    double root_min, root_max;
    int64_t n_p2p_pairs;     /* sum over target leaves of n_t * (points in its colleagues) */
    int64_t n_p2m_points;    /* source points entering P2M */
    int64_t n_m2l_pairs;     /* V-list (target box, source box) pairs */
    int64_t n_m2l_groups;    /* (target sibling group, parent direction) blocks with a source group */
    int64_t nodes_per_level[KIFMM_MAX_LEVELS];
    int64_t planned_bytes;   /* device memory of the planned-apply matrices (0 until built) */
} kifmm_tree_info;

/* Fill *o with the defaults listed above. */
void kifmm_default_options(kifmm_options *o);

/* FMM.__init__(x, y, kernel_functions, numba_functions, Nequiv, Ncutoff)
 * (class_fmm.py:167-176): a plan for one kernel, Nequiv equivalent/check
 * points per box and leaf cutoff Ncutoff.  No device work yet. */
int kifmm_plan_create(const kifmm_kernel *kernel, int32_t nequiv, int32_t ncutoff,
                      const kifmm_options *opts, kifmm_plan **plan_out);

/* FMM.build_tree() -> Tree(x, y, Ncutoff) (class_fmm.py:177-181, tree.py:464-522):
 * Morton keys, radix sort, leaf split, level restriction, X-list fake leaves,
 * colleague lists.  Points are copied; the caller keeps x, y. */
int kifmm_build_tree(kifmm_plan *plan, const double *x, const double *y, int64_t n, int32_t mem);

/* FMM.precompute() (class_fmm.py:182-298): per-level translation operators
 * in FP64 on the device, with the check-to-equivalent inverses composed in. */
int kifmm_precompute(kifmm_plan *plan);

/* FMM.build_expansions(tau) (class_fmm.py:299-352): P2M, M2M, M2L, L2L.
 * Every call starts from zeroed workspaces (a repeated apply is exact). */
int kifmm_build_expansions(kifmm_plan *plan, const double *tau, int32_t mem);

/* FMM.evaluate_to_points(x, y, check_self) at the plan's own source points
 * (class_fmm.py:379-399 with x, y the sources): L2P + P2P.  pot[n] is in
 * the caller's point order.  check_self skips pairs with equal coordinates
 * (class_fmm.py:107). */
int kifmm_evaluate_to_sources(kifmm_plan *plan, double *pot, int32_t check_self, int32_t mem);

/* FMM.evaluate_to_points(x, y, check_self) at arbitrary targets
 * (class_fmm.py:379-399): locate (tree.py:703-727), L2P, P2P. */
int kifmm_evaluate_to_points(kifmm_plan *plan, const double *x, const double *y, int64_t n,
                             int32_t check_self, double *pot, int32_t mem);

/* Wait for all work queued on the plan's stream, then report device-side
 * failures (a bounded wait in a kernel that ran out) as KIFMM_ERR_CUDA. */
int kifmm_synchronize(kifmm_plan *plan);

/* Repeated densities on one tree as one CUDA graph: the reference applies a
 * planned FMM to a new density with FMM.build_expansions(tau) followed by
 * FMM.evaluate_to_points(x, y, check_self) at the sources (class_fmm.py:299-352,
 * 379-399).  kifmm_graph_capture runs that pair once on the device pointers
 * tau_dev -> pot_dev (a normal apply, which allocates the plan's apply buffers),
 * then captures the same pair into a graph owned by the plan.
 * kifmm_graph_launch replays it on the plan's stream: it reads tau_dev as it is
 * when the replay runs and writes pot_dev; no host synchronisation, no
 * allocation.  The plan's stream must be a created stream (capture is not
 * possible on the legacy default stream).  build_tree or precompute on the plan
 * drops the graph.  Check results with kifmm_synchronize. */
int kifmm_graph_capture(kifmm_plan *plan, const double *tau_dev, double *pot_dev, int32_t check_self);
int kifmm_graph_launch(kifmm_plan *plan);

/* Packed applies of several plans (a serving batch): the same pair as
 * kifmm_graph_capture for plans[0..nplan), with the M2L of all plans in ONE
 * tensor-core launch and the near field + L2P of all plans in one launch per
 * kernel kind; the per-plan passes (P2M, M2M, L2L, gathers) run as parallel
 * branches of the graph.  Each plan's result is the same as its own apply
 * (the packed kernels run the same per-tile / per-leaf code on that plan's
 * data).  kifmm_batch_capture first runs one normal apply
 * (tau_dev[r] -> pot_dev[r]) of every plan that has not evaluated at its
 * sources since its tree and operators were built (that allocates the apply
 * buffers), then captures the packed graph without running it; each
 * kifmm_batch_launch computes every plan's apply from tau_dev[r] as it is
 * when the launch runs.  stream is the caller's created cudaStream_t on which
 * the capture and every launch are ordered.  Requirements: every plan precomputed, on
 * one device, distinct, in the mixed precision form with a tensor-core M2L
 * (one form for all), no near_fp64, planned or complex option; Laplace and
 * modified-Helmholtz plans may be mixed.  The plans must outlive the batch and
 * must not be rebuilt while it exists.  A batch holds the wait budget of its
 * plans at capture.  kifmm_batch_synchronize waits for the stream and reports
 * device-side failures of any plan as KIFMM_ERR_CUDA. */
typedef struct kifmm_batch kifmm_batch;
int kifmm_batch_capture(kifmm_plan *const *plans, int32_t nplan, const double *const *tau_dev,
                        double *const *pot_dev, int32_t check_self, void *stream, kifmm_batch **batch_out);
int kifmm_batch_launch(kifmm_batch *batch);
int kifmm_batch_synchronize(kifmm_batch *batch);
/* Densities drawn by the batch itself: before the next kifmm_batch_launch,
 * lane r gets tau_dev[r] = N(0,1) density number index[r] of seed seed[r]
 * (the values of kifmm_fill_normal(tau_dev[r], n_r, seed[r], index[r])), drawn
 * by the graph's first kernel; seed[r] = UINT64_MAX leaves tau_dev[r] as the
 * caller wrote it.  The setting holds for later launches until changed. */
int kifmm_batch_set_draws(kifmm_batch *batch, const uint64_t *seed, const uint64_t *index);
/* After kifmm_batch_synchronize: sums[r] = sum of pot_dev[r] of the last launch
 * (summed on the device by the graph's last kernel, in a fixed order). */
int kifmm_batch_sums(kifmm_batch *batch, double *sums);
/* Tiles of the packed M2L launch and leaves of the packed leaf launches. */
int kifmm_batch_info(kifmm_batch *batch, int64_t *m2l_tiles, int64_t *leaves);
int kifmm_batch_destroy(kifmm_batch *batch);

/* A new non-blocking cudaStream_t on `device` (for hosts without a CUDA
 * runtime binding of their own, e.g. a server that needs streams no other
 * library hands out), and its release. */
int kifmm_stream_create(int32_t device, void **stream);
int kifmm_stream_destroy(void *stream);

/* out[0..n) = N(0,1) density number `index` of stream `seed` (seed != UINT64_MAX),
 * from a counter-based generator (Philox4x32-10 + Box-Muller): the values
 * depend only on (seed, index, position), not on the launch that draws them.
 * out is a device pointer; work is ordered on the cudaStream_t `stream`. */
int kifmm_fill_normal(double *out, int64_t n, uint64_t seed, uint64_t index, void *stream);

/* Tree statistics (reference Tree.levels, Level.n_node, ...). */
int kifmm_get_tree_info(kifmm_plan *plan, kifmm_tree_info *info);

/* Canonical tree for parity checks: nodes[n_nodes][7] = (level, ix, iy,
 * leaf, fake_leaf, Xlist, ns) with ix = (xmin - root_min)/width, in the same
 * meaning as the reference's Level arrays (tree.py:313-420); point_leaf[n][3]
 * = (level, ix, iy) of the leaf holding each point (tree.py:703-727).
 * Host buffers; either may be NULL. */
int kifmm_export_tree(kifmm_plan *plan, int64_t *nodes, int64_t *point_leaf);

/* Interaction lists for parity checks, with node numbers = rows of
 * kifmm_export_tree's nodes array (host buffers, each may be NULL):
 *   colleagues[n_nodes][9]: the same-level colleague at cell offset (dx, dy)
 *     in slot (dx+1)*3 + (dy+1), -1 if none -- the reference's Level.colleagues
 *     (tree.py:349-375) ordered by direction;
 *   m2l[*n_m2l][2]: (target, source) node pairs of every M2L translation the
 *     apply performs: the children of each split cell receive, from each
 *     colleague's child group that holds points, every well-separated child --
 *     the reference's numba_add_interactions blocks (class_fmm.py:17-33,
 *     :323-343) except those into the fake children of X-list leaves, whose
 *     local expansions the reference computes but never reads;
 *   p2p[*n_p2p][2]: (leaf, source) node pairs of the near field: each leaf
 *     holding points reads every colleague holding points
 *     (numba_target_neighbor_evaluation, class_fmm.py:90-111).
 * n_m2l / n_p2p receive the pair counts; when m2l / p2p is given, the count
 * pointer must hold its capacity in pairs on entry (KIFMM_ERR_ARG if short). */
int kifmm_export_lists(kifmm_plan *plan, int64_t *colleagues, int64_t *m2l, int64_t *n_m2l, int64_t *p2p,
                       int64_t *n_p2p);

/* Release the plan and its device memory. */
int kifmm_plan_destroy(kifmm_plan *plan);

/* Text of the calling thread's last error ("" if none). */
const char *kifmm_last_error(void);

/* Get_Kernel_Functions(...).KAS (class_fmm.py:134-143), restricted to chosen
 * targets: FP64 direct sum out[a] = sum_{i != t_a} G(s_i -> s_{t_a}) tau_i.
 * The O(N^2) oracle of the error metric, on the GPU. */
int kifmm_direct_sum(const kifmm_kernel *kernel, const double *x, const double *y,
                     const double *tau, int64_t n, const int64_t *targets, int64_t nt,
                     double *out, int32_t mem, int32_t device);

/* Get_Kernel_Functions(...).KF (class_fmm.py:116-122) / Kernel_Form
 * (:147-164): out[j*ns + i] = G(s_i -> t_j), FP64. */
int kifmm_kernel_matrix(const kifmm_kernel *kernel, const double *sx, const double *sy, int64_t ns,
                        const double *tx, const double *ty, int64_t nt, double *out,
                        int32_t mem, int32_t device);

/* Get_Kernel_Functions(...).KA (class_fmm.py:124-132): out[j] =
 * sum_i G(s_i -> t_j) tau_i, FP64. */
int kifmm_kernel_apply(const kifmm_kernel *kernel, const double *sx, const double *sy, int64_t ns,
                       const double *tx, const double *ty, int64_t nt, const double *tau,
                       double *out, int32_t mem, int32_t device);

/* Phase timers (no counterpart in the reference, which prints wall-clock
 * phase times when verbose, class_fmm.py:178-181,297-298,320-352).  When
 * enabled, CUDA events on the plan's stream bracket each phase and the device
 * milliseconds accumulate per phase id (KIFMM_PHASE_*). */
enum {
    KIFMM_PHASE_TREE = 0,      /* whole build_tree */
    KIFMM_PHASE_SORT = 1,      /* Morton radix sort of the points (inside TREE) */
    KIFMM_PHASE_PRECOMPUTE = 2, /* wait for the operators (started by build_tree) */
    KIFMM_PHASE_P2M = 3,
    KIFMM_PHASE_M2M = 4,
    KIFMM_PHASE_M2L = 5,       /* M2L, all levels (with L2L where one kernel does both) */
    KIFMM_PHASE_LEAF = 6,      /* L2P + P2P at the sources */
    KIFMM_PHASE_TARGETS = 7,   /* locate + L2P + P2P at separate targets */
    KIFMM_PHASE_L2L = 8,       /* separate L2L chain (after the tensor-core M2L) */
    KIFMM_PHASE_OPERATORS = 9, /* operator construction on the side stream, overlapping TREE */
    KIFMM_PHASE_CLOSURE = 10,  /* split cells, level restriction, X-list (inside TREE) */
    KIFMM_PHASE_ENTRIES = 11,  /* sort of the split-cell entries (inside TREE) */
    KIFMM_PHASE_NODES = 12,    /* node tables and work lists (inside TREE) */
    KIFMM_PHASE_COUNT = 13
};
int kifmm_set_profiling(kifmm_plan *plan, int32_t on);
/* ms[KIFMM_PHASE_COUNT] and launches[KIFMM_PHASE_COUNT] (either may be NULL);
 * reset != 0 clears the accumulators after reading. */
int kifmm_get_phase_times(kifmm_plan *plan, double *ms, int64_t *launches, int32_t reset);

/* Poll budget of the bounded waits inside the apply kernels (no counterpart
 * in the reference, which has no device code): the bulk-copy waits of the
 * M2M/L2L level kernels and the copy/MMA completion waits of the tensor-core
 * M2L.  A wait that runs out sets a device error flag; the kernel then waits
 * for its own copies and MMAs in flight (with a fixed budget), frees what it
 * holds and returns, and the next kifmm_synchronize (or host-buffer
 * evaluation) on the plan reports KIFMM_ERR_CUDA.  polls >= 0 sets the budget
 * (0: every first wait runs out at once, which tests that path); polls < 0
 * restores the default.  Drops a captured graph. */
int kifmm_set_wait_limit(kifmm_plan *plan, int64_t polls);

/* Number of kernels this library has launched in the process so far. */
int64_t kifmm_launch_count(void);

/* No counterpart in the reference (it has no device memory at all).
 * For callers that cannot call cudaMalloc -- code running where another
 * component owns all device memory, or a loop that must not enter the
 * allocator: the first stage of the tree build, allocating nothing.
 * keys[i] = 58-bit Morton key (x bit above y bit) of the i-th point in
 * sorted order on the 2^29 x 2^29 grid of the root box [root_min, root_max]
 * (integer corners, as kifmm_get_tree_info reports; points outside the box
 * clamp to its edge cells; a non-finite coordinate gives key 0 -- this call
 * does not check its input the way kifmm_build_tree does), perm[i] = index of
 * that point in x, y.  The sort is stable.  x, y, keys, perm are device
 * pointers on the current device; work is queued on `stream` (NULL: the
 * legacy default stream) and the call returns before it finishes.  Scratch is
 * one fixed device array of the library (about 12.3 MB), so n may not exceed
 * KIFMM_NOALLOC_MAX_POINTS.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress).  CUDA loads modules lazily by default, so
 * that first call is also when the array is allocated on the device: make it
 * before the host hands all device memory to its own pool and before any
 * stream capture (or set CUDA_MODULE_LOADING=EAGER, which reserves the array
 * on every device when the library loads).  From then on the device holds the
 * array until the process exits; the cached address does not survive
 * cudaDeviceReset.  All calls share the array: calls whose work overlaps on
 * the GPU (other streams, other threads) race. */
#define KIFMM_NOALLOC_MAX_POINTS 1048576
int kifmm_morton_sort_noalloc(const double *x, const double *y, int64_t n, double root_min, double root_max,
                              uint64_t *keys, int32_t *perm, void *stream);

/* Library version (major*10000 + minor*100 + patch). */
int kifmm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* KIFMM2D_H */
