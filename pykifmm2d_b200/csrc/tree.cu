// tree.cu -- level-restricted adaptive quadtree on the GPU.
//
// Reference: Tree (pykifmm2d/tree.py:460-590).  The reference splits level by
// level with in-place partitions; here the same tree is derived from sorted
// Morton keys:
//   * root box [m, M] as in tree.py:475-484 (including its ymax = y.min()
//     quirk unless fix_bbox), all midpoints exact dyadic numbers, so the
//     reference's strict 'x > xmid' descent equals the key prefix;
//   * a cell is split in the unrestricted tree iff it holds > Ncutoff points
//     (tree.py:242): found from the sorted keys in one pass -- point i reports
//     the cells it opens whose window [i, i+Ncutoff] stays inside them;
//   * level restriction (tree.py:533-545, numba_get_bads :432-444) is the
//     closure Split_l = Split0_l U N9(parent(Split_{l+1})) (N9 = the 3x3
//     block of cells in the domain), built by chains of rectangles from the
//     T0 cells in one launch (k_closure);
//   * X-list (tree.py:546-576, numba_get_Xlist :446-458): a real leaf with a
//     split colleague gets four fake children;
//   * nodes of level l+1 are the four children of every split or X-list cell
//     of level l, in Morton order; colleagues (tree.py:260-294) are the
//     existing same-level cells of the 3x3 block, stored by direction.
// Split and X-list cells live in a device hash set; once collected they are
// sorted into one list, and lookups probe the table, which maps each entry to
// its sorted position (k_hash_index).
#include <algorithm>
#include <cmath>
#include <cstring>

#include <optional>

#include "kifmm_internal.cuh"

namespace kifmm {
void build_leaf_records(kifmm_plan *P);  // passes.cu
void build_m2l_order(kifmm_plan *P);     // passes.cu
}

namespace kifmm {

constexpr uint64_t KEY56 = (1ull << 56) - 1;

__device__ __forceinline__ uint64_t ordered_bits(double v) {
    uint64_t u = (uint64_t)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double from_ordered(uint64_t o) {
    uint64_t u = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    double d;
    memcpy(&d, &u, 8);
    return d;
}

// Root box from the ordered extremes in scal[0..3] (tree.py:475-484, with the
// reference's ymax = y.min() unless fix_bbox): m = floor(min(xmin, ymin)),
// M = ceil(max(xmax, ytop)).  Computed the same way on the device (k_keys_dev)
// and on the host once the counts come back.
__host__ __device__ inline void root_box(const unsigned long long *sc, int fix_bbox, double &m, double &M) {
    const double xmn = from_ordered(sc[0]), xmx = from_ordered(sc[1]), ymn = from_ordered(sc[2]),
                 ymx = from_ordered(sc[3]);
    const double ytop = fix_bbox ? ymx : ymn;
    m = floor(fmin(xmn, ymn));
    M = ceil(fmax(xmx, ytop));
}

// scal[0..3]: ordered min x, max x, min y, max y; scal[4]: non-finite count
__global__ void k_bbox(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                       unsigned long long *scal) {
    uint64_t mnx = ~0ull, mxx = 0, mny = ~0ull, mxy = 0;
    unsigned long long bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double a = x[i], b = y[i];
        if (!isfinite(a) || !isfinite(b)) { bad++; continue; }
        uint64_t oa = ordered_bits(a), ob = ordered_bits(b);
        mnx = min(mnx, oa); mxx = max(mxx, oa);
        mny = min(mny, ob); mxy = max(mxy, ob);
    }
    for (int o = 16; o; o >>= 1) {
        mnx = min(mnx, (uint64_t)__shfl_xor_sync(0xffffffffu, mnx, o));
        mxx = max(mxx, (uint64_t)__shfl_xor_sync(0xffffffffu, mxx, o));
        mny = min(mny, (uint64_t)__shfl_xor_sync(0xffffffffu, mny, o));
        mxy = max(mxy, (uint64_t)__shfl_xor_sync(0xffffffffu, mxy, o));
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    // one global atomic per value and block (not per warp: they all hit the same words)
    __shared__ unsigned long long red[5][32];
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = mnx; red[1][w] = mxx; red[2][w] = mny; red[3][w] = mxy; red[4][w] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < nw; i++) {
            mnx = min(mnx, (uint64_t)red[0][i]); mxx = max(mxx, (uint64_t)red[1][i]);
            mny = min(mny, (uint64_t)red[2][i]); mxy = max(mxy, (uint64_t)red[3][i]);
            bad += red[4][i];
        }
        atomicMin(&scal[0], mnx); atomicMax(&scal[1], mxx);
        atomicMin(&scal[2], mny); atomicMax(&scal[3], mxy);
        if (bad) atomicAdd(&scal[4], bad);
    }
}

// Exact grid cell: j = #{k in [1, 2^D-1] : v > m + k h}.  The gridlines are
// the midpoints of every level (m + odd * W / 2^(l+1)), exact in FP64 for the
// coordinate range checked on the host.
__device__ __forceinline__ uint64_t grid_cell(double v, double m, double h) {
    const int64_t top = (1ll << KEY_DEPTH) - 1;
    double t = ceil((v - m) / h) - 1.0;
    int64_t j = t < 0 ? 0 : (t > (double)top ? top : (int64_t)t);
    for (int it = 0; it < 8 && j < top && v > m + (double)(j + 1) * h; it++) j++;
    for (int it = 0; it < 8 && j > 0 && !(v > m + (double)j * h); it++) j--;
    return (uint64_t)j;
}

__global__ void k_keys(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double m, double M,
                       double h, uint64_t *__restrict__ key, int32_t *__restrict__ perm, unsigned long long *outside) {
    unsigned long long out = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double a = x[i], b = y[i];
        uint64_t k = 0;
        if (h > 0 && isfinite(a) && isfinite(b)) k = morton(grid_cell(a, m, h), grid_cell(b, m, h));
        key[i] = k;
        perm[i] = (int32_t)i;
        out += (a < m || a > M || b < m || b > M);
    }
    if (!outside) return;
    for (int o = 16; o; o >>= 1) out += __shfl_xor_sync(0xffffffffu, out, o);
    if ((threadIdx.x & 31) == 0 && out) atomicAdd(outside, out);
}

// Separate targets in the Morton order of the plan's root box, so that the
// targets of one warp mostly share a leaf (its node tables and near sources
// are then read once per warp, not once per lane): keys of the coordinates
// clamped into the box, a sort by the top 32 key bits (16 levels), and the
// coordinates gathered in that order.  Non-finite coordinates get key 0.
__global__ void k_target_keys(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double m,
                              double h, uint64_t *__restrict__ key, int32_t *__restrict__ perm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double a = x[i], b = y[i];
        key[i] = (h > 0 && isfinite(a) && isfinite(b)) ? morton(grid_cell(a, m, h), grid_cell(b, m, h)) : 0;
        perm[i] = (int32_t)i;
    }
}

__global__ void k_gather2(const double *__restrict__ x, const double *__restrict__ y, const int32_t *__restrict__ perm,
                          int64_t n, double *__restrict__ xs, double *__restrict__ ys);

void sort_targets(kifmm_plan *P, const double *tx, const double *ty, int64_t n) {
    KIFMM_REQUIRE(n < (1ll << 31), KIFMM_ERR_ARG, "evaluate_to_points: more than 2^31 - 1 targets");
    P->tkey.alloc(n); P->tkey2.alloc(n); P->tperm.alloc(n); P->tperm2.alloc(n);
    P->txs.alloc(n); P->tys.alloc(n);
    cudaStream_t s = P->stream;
    const unsigned gs = grid_for(n, 256, P->num_sms * 8);
    k_target_keys<<<gs, 256, 0, s>>>(tx, ty, n, P->root_min, std::ldexp(P->W, -KEY_DEPTH), P->tkey.p, P->tperm.p);
    KIFMM_LAUNCHED();
    radix_sort_pairs_bits(P->tkey.p, P->tperm.p, P->tkey2.p, P->tperm2.p, n, 2 * KEY_DEPTH - 32, 32, P);
    launch_pdl(k_gather2, dim3(gs), dim3(256), 0, s, tx, ty, (const int32_t *)P->tperm.p, n, P->txs.p, P->tys.p);
}

// k_keys with the root box read from the device (no host round trip after
// k_bbox).  Inputs that the host will reject (non-finite coordinates, |m| or
// |M| >= 2^23) get key 0 here; the host reports them at its next read-back.
__global__ void k_keys_dev(const double *__restrict__ x, const double *__restrict__ y, int64_t n, int fix_bbox,
                           const unsigned long long *__restrict__ scal, uint64_t *__restrict__ key,
                           int32_t *__restrict__ perm, unsigned long long *outside) {
    pdl_trigger();
    pdl_wait();
    double m, M;
    root_box(scal, fix_bbox, m, M);
    const bool valid = scal[4] == 0 && fabs(m) < 8388608.0 && fabs(M) < 8388608.0;
    const double h = (valid && M > m) ? ldexp(M - m, -KEY_DEPTH) : 0.0;
    unsigned long long out = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double a = x[i], b = y[i];
        uint64_t k = 0;
        if (h > 0 && isfinite(a) && isfinite(b)) k = morton(grid_cell(a, m, h), grid_cell(b, m, h));
        key[i] = k;
        perm[i] = (int32_t)i;
        out += (a < m || a > M || b < m || b > M);
    }
    for (int o = 16; o; o >>= 1) out += __shfl_xor_sync(0xffffffffu, out, o);
    if ((threadIdx.x & 31) == 0 && out) atomicAdd(outside, out);
}

__global__ void k_gather2(const double *__restrict__ x, const double *__restrict__ y, const int32_t *__restrict__ perm,
                          int64_t n, double *__restrict__ xs, double *__restrict__ ys) {
    pdl_trigger();
    pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = perm[i];
        xs[i] = x[p];
        ys[i] = y[p];
    }
}

// deepest level whose cell contains both keys
__device__ __forceinline__ int common_level(uint64_t a, uint64_t b) {
    if (a == b) return KEY_DEPTH;
    return (__clzll((long long)(a ^ b)) - (64 - 2 * KEY_DEPTH)) >> 1;
}

// ------------------------------------------------------------ hash set
__device__ __forceinline__ uint64_t hmix(uint64_t v) {
    v ^= v >> 33; v *= 0xff51afd7ed558ccdull;
    v ^= v >> 33; v *= 0xc4ceb9fe1a85ec53ull;
    v ^= v >> 33;
    return v;
}

struct HashSet {
    unsigned long long *tab;
    uint64_t mask;
    uint64_t *list;
    unsigned long long *count;  // entries appended to list
    unsigned long long *ovf;
    uint64_t cap;               // list capacity
    unsigned long long *lcount; // [32] entries per level, counted as they are appended
};

__device__ __forceinline__ uint64_t ent_make(int l, uint64_t k, int x) {
    return ((uint64_t)l << ENT_LEVEL_SHIFT) | (k << 1) | (uint64_t)x;
}

// Claim entry e in the table: true iff this call stored it (the caller then
// appends it to the list).  A plain read comes first, so that the many probes
// of cells that are already in the set take no atomic.
__device__ __forceinline__ bool hs_claim(const HashSet &H, uint64_t e) {
    uint64_t s = hmix(e) & H.mask;
    for (uint64_t p = 0; p <= H.mask; p++) {
        const uint64_t v = ((volatile unsigned long long *)H.tab)[s];
        if (v == e) return false;
        if (v == ENT_EMPTY) {
            const unsigned long long prev = atomicCAS(&H.tab[s], (unsigned long long)ENT_EMPTY, (unsigned long long)e);
            if (prev == ENT_EMPTY) return true;
            if (prev == e) return false;
        }
        s = (s + 1) & H.mask;
    }
    atomicOr(H.ovf, 2ull);
    return false;
}

__device__ bool hs_has(const HashSet &H, uint64_t e) {
    uint64_t s = hmix(e) & H.mask;
    for (uint64_t p = 0; p <= H.mask; p++) {
        uint64_t v = ((volatile unsigned long long *)H.tab)[s];
        if (v == e) return true;
        if (v == ENT_EMPTY) return false;
        s = (s + 1) & H.mask;
    }
    return false;
}

// Append the claimed entries of a warp (lanes in `fm`, all of level l) with
// one atomic on the list count and one on the level count.
__device__ __forceinline__ void warp_append(const HashSet &H, unsigned fm, uint64_t e, int l, int lane) {
    if (!fm) return;
    const int lead = __ffs(fm) - 1;
    unsigned long long base = 0;
    if (lane == lead) {
        base = atomicAdd(H.count, (unsigned long long)__popc(fm));
        atomicAdd(&H.lcount[l], (unsigned long long)__popc(fm));
    }
    base = __shfl_sync(0xffffffffu, base, lead);
    if ((fm >> lane) & 1) {
        const unsigned long long idx = base + __popc(fm & ((1u << lane) - 1));
        if (idx < H.cap) H.list[idx] = e;
        else atomicOr(H.ovf, 1ull);
    }
}

// Split cells of the unrestricted tree (T0).  Point i (sorted) is the first
// point of its level-l cell for l > common_level(key[i-1], key[i]); that cell
// holds more than ppl points iff l <= common_level(key[i], key[i+ppl]).
// Counting pass: scal[5] cell count, scal[6] deepest split level + 1,
// scal[7] depth overflow.
__global__ void k_t0_count(const uint64_t *__restrict__ key, int64_t n, int64_t ppl, unsigned long long *scal) {
    pdl_trigger();
    pdl_wait();
    unsigned long long cnt = 0;
    int deepest = 0;
    bool over = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i + ppl >= n) continue;
        uint64_t k = key[i];
        int hi = common_level(k, key[i + ppl]);
        if (hi >= KEY_DEPTH) { over = true; hi = KEY_DEPTH - 1; }
        int lo = i == 0 ? -1 : common_level(key[i - 1], k);
        if (hi <= lo) continue;
        cnt += (unsigned long long)(hi - lo);
        deepest = max(deepest, hi + 1);
    }
    for (int o = 16; o; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        deepest = max(deepest, __shfl_xor_sync(0xffffffffu, deepest, o));
    }
    over = __any_sync(0xffffffffu, over);
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(&scal[5], cnt);
        atomicMax(&scal[6], (unsigned long long)deepest);
        if (over) atomicOr(&scal[7], 1ull);
    }
}

// Level restriction (tree.py:533-545) as chains instead of a level-by-level
// sweep.  The restricted set is the smallest S containing T0 with
// N9(parent(x)) in S for every x in S (N9 = the 3x3 block of cells in the
// domain).  N9 o parent maps a rectangle of cells to a rectangle (at most
// 5 x 5: widths w -> w/2 + 2 settle at 4) and distributes over unions, so the
// set is built by chains: the chain of T0 cell x inserts R = N9(parent(x)),
// then N9(parent(R)), ..., and stops after a level where it stored nothing new.
// That is complete: every cell of S was stored first either by T0 (and then
// has its own chain) or by a chain, which then went on one level with a
// rectangle containing the cell's N9(parent).  One warp runs a chain, a lane
// per cell of the rectangle.
__device__ void t0_chain(const HashSet &H, int l0, uint64_t c0, int lane) {
    {
        const uint64_t e = ent_make(l0, c0, 0);
        const bool fresh = lane == 0 && hs_claim(H, e);
        warp_append(H, __ballot_sync(0xffffffffu, fresh), e, l0, lane);
    }
    int64_t x0 = (int64_t)compact2(c0 >> 1), y0 = (int64_t)compact2(c0), x1 = x0, y1 = y0;
    for (int l = l0 - 1; l >= 0; l--) {
        const int64_t top = (1ll << l) - 1;
        x0 = max((x0 >> 1) - 1, (int64_t)0); x1 = min((x1 >> 1) + 1, top);
        y0 = max((y0 >> 1) - 1, (int64_t)0); y1 = min((y1 >> 1) + 1, top);
        const int w = (int)(x1 - x0 + 1), h = (int)(y1 - y0 + 1);
        uint64_t e = 0;
        bool fresh = false;
        if (lane < w * h) {
            const int64_t cx = x0 + lane % w, cy = y0 + lane / w;
            e = ent_make(l, morton((uint64_t)cx, (uint64_t)cy), 0);
            fresh = hs_claim(H, e);
        }
        const unsigned fm = __ballot_sync(0xffffffffu, fresh);
        warp_append(H, fm, e, l, lane);
        if (!fm) break;
    }
}

// T0 cells and their restriction chains: one warp per 32 sorted points; each
// point that opens split cells (levels lo+1..hi) runs their chains, deepest
// first, so that the chains of its coarser cells mostly find their cells in
// the set and stop after one level.
__global__ void __launch_bounds__(256) k_closure(const uint64_t *__restrict__ key, int64_t n, int64_t ppl,
                                                 HashSet H) {
    pdl_trigger();
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w * 32 + ppl < n; w += nw) {
        const int64_t i = w * 32 + lane;
        int lo = 0, hi = -1;
        uint64_t k = 0;
        if (i + ppl < n) {
            k = key[i];
            hi = min(common_level(k, key[i + ppl]), KEY_DEPTH - 1);
            lo = i == 0 ? -1 : common_level(key[i - 1], k);
        }
        for (unsigned om = __ballot_sync(0xffffffffu, hi > lo); om; om &= om - 1) {
            const int src = __ffs(om) - 1;
            const uint64_t ks = __shfl_sync(0xffffffffu, k, src);
            const int los = __shfl_sync(0xffffffffu, lo, src), his = __shfl_sync(0xffffffffu, hi, src);
            for (int l = his; l > los; l--) t0_chain(H, l, ks >> (2 * (KEY_DEPTH - l)), lane);
        }
    }
}

__device__ __forceinline__ unsigned long long hs_count(const HashSet &H) {
    unsigned long long n = *((volatile unsigned long long *)H.count);
    return n > H.cap ? H.cap : n;
}

// X-list (tree.py:546-576, numba_get_Xlist :446-458): for levels 1..L-2, a
// real leaf (cell not split, parent split) next to a split cell becomes an
// X-list cell (every split cell lies on a level <= L-2, so the level range
// follows from the split cells themselves).  One item per (split cell, neighbour); the warp's new cells are
// appended together (one count atomic per warp, one level atomic per level).
__global__ void __launch_bounds__(256) k_xlist(HashSet H) {
    pdl_trigger();
    pdl_wait();
    const unsigned long long n = hs_count(H);
    const int lane = threadIdx.x & 31;
    const int64_t total = 9 * (int64_t)n, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) & ~(int64_t)31; base < total;
         base += stride) {
        const int64_t j = base + lane;
        bool fresh = false;
        uint64_t e = 0;
        int l = 0;
        if (j < total) {
            const int64_t i = j / 9;
            const int d = (int)(j - 9 * i);
            const uint64_t s = H.list[i];
            l = (int)(s >> ENT_LEVEL_SHIFT);
            if (d != 4 && !(s & 1) && l >= 1) {  // split cells lie on levels <= L-2
                const uint64_t k = (s >> 1) & KEY56;
                const int64_t cx = (int64_t)compact2(k >> 1) + d / 3 - 1, cy = (int64_t)compact2(k) + d % 3 - 1;
                const int64_t side = 1ll << l;
                if (cx >= 0 && cy >= 0 && cx < side && cy < side) {
                    const uint64_t c = morton((uint64_t)cx, (uint64_t)cy);
                    if (!hs_has(H, ent_make(l, c, 0)) && hs_has(H, ent_make(l - 1, c >> 2, 0))) {
                        e = ent_make(l, c, 1);
                        fresh = hs_claim(H, e);
                    }
                }
            }
        }
        const unsigned fm = __ballot_sync(0xffffffffu, fresh);
        if (!fm) continue;
        const int lead = __ffs(fm) - 1;
        unsigned long long b0 = 0;
        if (lane == lead) b0 = atomicAdd(H.count, (unsigned long long)__popc(fm));
        b0 = __shfl_sync(0xffffffffu, b0, lead);
        if (fresh) {
            const unsigned peers = __match_any_sync(fm, l);
            if (lane == __ffs(peers) - 1) atomicAdd(&H.lcount[l], (unsigned long long)__popc(peers));
            const unsigned long long idx = b0 + __popc(fm & ((1u << lane) - 1));
            if (idx < H.cap) H.list[idx] = e;
            else atomicOr(H.ovf, 1ull);
        }
    }
}

// ----------------------------------------------------------- node arrays
// Entry lookup by hash probe: the split-cell set's table holds every entry
// (with its X-list bit), and hidx[slot] is the sorted position of the entry in
// that slot (k_hash_index).  One or two probes instead of a binary search.
struct EntryIndex {
    const unsigned long long *tab;
    const int32_t *hidx;
    uint64_t mask;
};
__device__ __forceinline__ int64_t find_entry_h(const EntryIndex &X, int l, uint64_t k) {
    if (l < 0 || !X.hidx) return -1;  // no entries (single-leaf tree): no table either
    for (int x = 0; x < 2; x++) {
        const uint64_t e = ent_make(l, k, x);
        uint64_t s = hmix(e) & X.mask;
        for (uint64_t p = 0; p <= X.mask; p++) {
            const uint64_t v = X.tab[s];
            if (v == e) return X.hidx[s];
            if (v == ENT_EMPTY) break;
            s = (s + 1) & X.mask;
        }
    }
    return -1;
}
__device__ __forceinline__ int64_t node_index_h(const EntryIndex &X, const LevelTable &T, int l, uint64_t k) {
    if (l == 0) return k == 0 ? 0 : -1;
    int64_t j = find_entry_h(X, l - 1, k >> 2);
    if (j < 0) return -1;
    return T.off[l] + 4 * (j - T.eoff[l - 1]) + (int64_t)(k & 3);
}
__global__ void k_hash_index(const uint64_t *__restrict__ ent, int64_t n_ent, const unsigned long long *__restrict__ tab,
                             uint64_t mask, int32_t *__restrict__ hidx) {
    pdl_trigger();
    pdl_wait();
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n_ent; j += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t e = ent[j];
        uint64_t s = hmix(e) & mask;
        for (uint64_t p = 0; p <= mask; p++) {
            if (tab[s] == e) {
                hidx[s] = (int32_t)j;
                break;
            }
            s = (s + 1) & mask;
        }
    }
}

__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t *__restrict__ a, int64_t n, uint64_t v) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void k_nodes(LevelTable T, EntryIndex X, int64_t n_nodes, const uint64_t *__restrict__ ent,
                        const uint64_t *__restrict__ pkey, int64_t npts, uint64_t *__restrict__ nkey,
                        int8_t *__restrict__ nlev, uint8_t *__restrict__ nflag, int32_t *__restrict__ nbot,
                        int32_t *__restrict__ ntop, int32_t *__restrict__ nparent, int32_t *__restrict__ nchild,
                        int32_t *__restrict__ nent, int32_t *__restrict__ ncoll, int32_t *__restrict__ ent_node) {
    pdl_trigger();
    pdl_wait();
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_nodes; g += (int64_t)gridDim.x * blockDim.x) {
        int l = 0;
        while (l + 1 < T.L && T.off[l + 1] <= g) l++;
        int64_t i = g - T.off[l];
        uint64_t k = 0;
        uint8_t f = 0;
        int64_t parent = -1;
        if (l > 0) {
            uint64_t pe = ent[T.eoff[l - 1] + i / 4];
            uint64_t pk = (pe >> 1) & KEY56;
            k = (pk << 2) | (uint64_t)(i & 3);
            if (pe & 1) f |= NF_FAKE;
            parent = node_index_h(X, T, l - 1, pk);
        }
        int64_t j = find_entry_h(X, l, k);
        int64_t child = -1;
        if (j >= 0) {
            f |= (ent[j] & 1) ? NF_XLIST : NF_SPLIT;
            child = T.off[l + 1] + 4 * (j - T.eoff[l]);
            ent_node[j] = (int32_t)g;
        }
        int sh = 2 * (KEY_DEPTH - l);
        uint64_t lo = k << sh;
        int64_t b = l == 0 ? 0 : lower_bound_u64(pkey, npts, lo);
        int64_t e = (l == 0) ? npts : lower_bound_u64(pkey, npts, lo + (1ull << sh));
        nkey[g] = k;
        nlev[g] = (int8_t)l;
        nflag[g] = f;
        nbot[g] = (int32_t)b;
        ntop[g] = (int32_t)e;
        nparent[g] = (int32_t)parent;
        nchild[g] = (int32_t)child;
        nent[g] = (int32_t)j;
        int64_t ix = (int64_t)compact2(k >> 1), iy = (int64_t)compact2(k), side = 1ll << l;
        for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++) {
                int64_t cx = ix + dx, cy = iy + dy, c = -1;
                if (cx >= 0 && cy >= 0 && cx < side && cy < side)
                    c = (dx == 0 && dy == 0) ? g : node_index_h(X, T, l, morton((uint64_t)cx, (uint64_t)cy));
                ncoll[9 * g + (dx + 1) * 3 + (dy + 1)] = (int32_t)c;
            }
    }
}

// Work lists in node order (level-major, Morton order within a level), so
// that consecutive entries share a level and a neighbourhood.  The nodes are
// cut into tiles of LT_TILE: k_lists_count counts each tile's entries,
// k_lists_scan turns the counts into offsets, k_lists_write compacts each
// tile in order.  cnt: [0] leaf_list, [1] p2m_list, [2] leaves, [3] fake,
// [4] xlist.
constexpr int LT_THREADS = 256, LT_TILE = LT_THREADS * 2;  // ~300 blocks for 150k nodes
struct ListFlags {
    bool leaf = false, p2m = false, real_leaf = false, fake = false, xl = false;
};
__device__ __forceinline__ ListFlags list_flags(int64_t g, const int8_t *nlev, const uint8_t *nflag,
                                                const int32_t *nbot, const int32_t *ntop) {
    ListFlags r;
    const uint8_t f = nflag[g];
    r.fake = f & NF_FAKE;
    r.xl = f & NF_XLIST;
    r.real_leaf = !r.fake && !(f & NF_SPLIT);
    const bool pts = ntop[g] > nbot[g];
    r.leaf = r.real_leaf && pts;
    r.p2m = nlev[g] >= 2 && pts && ((r.real_leaf && !r.xl) || r.fake);
    return r;
}
// Exclusive scan over the block (blockDim.x a multiple of 32); total = block sum.
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned *sm, unsigned &total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned z = lane < nw ? sm[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        sm[lane] = z;  // inclusive prefix of the warp sums
    }
    __syncthreads();
    const unsigned r = (wid ? sm[wid - 1] : 0u) + x - v;
    total = sm[nw - 1];
    __syncthreads();
    return r;
}
// lcnt[l]: entries of leaf_list on level l (leaf_list is level-major, so they
// are the contiguous range after those of the levels above)
__global__ void __launch_bounds__(LT_THREADS) k_lists_count(int64_t n_nodes, const int8_t *__restrict__ nlev,
                                                            const uint8_t *__restrict__ nflag,
                                                            const int32_t *__restrict__ nbot,
                                                            const int32_t *__restrict__ ntop, uint32_t *tcnt,
                                                            unsigned long long *cnt, unsigned long long *lcnt) {
    pdl_trigger();
    pdl_wait();
    __shared__ unsigned sm[32];
    __shared__ unsigned slv[MAX_LEVELS];
    if (threadIdx.x < MAX_LEVELS) slv[threadIdx.x] = 0;
    __syncthreads();
    const int64_t g0 = (int64_t)blockIdx.x * LT_TILE;
    unsigned c[5] = {0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < LT_TILE; i += LT_THREADS) {
        const int64_t g = g0 + i;
        if (g >= n_nodes) break;
        const ListFlags f = list_flags(g, nlev, nflag, nbot, ntop);
        c[0] += f.leaf;
        c[1] += f.p2m;
        c[2] += f.real_leaf;
        c[3] += f.fake;
        c[4] += f.xl;
        if (f.leaf) atomicAdd(&slv[nlev[g]], 1u);
    }
    __syncthreads();
    if (threadIdx.x < MAX_LEVELS && slv[threadIdx.x]) atomicAdd(&lcnt[threadIdx.x], (unsigned long long)slv[threadIdx.x]);
#pragma unroll
    for (int k = 0; k < 5; k++) {
        unsigned t;
        block_excl_scan(c[k], sm, t);
        if (threadIdx.x == 0) {
            if (k < 2) tcnt[2 * blockIdx.x + k] = t;
            else if (t) atomicAdd(&cnt[k], (unsigned long long)t);
        }
    }
}
// one block: tile counts -> exclusive tile offsets (both lists); totals to cnt[0..1]
__global__ void __launch_bounds__(1024) k_lists_scan(int64_t ntiles, uint32_t *tcnt, unsigned long long *cnt) {
    pdl_trigger();
    pdl_wait();
    __shared__ unsigned sm[32];
    unsigned carry0 = 0, carry1 = 0;
    for (int64_t base = 0; base < ntiles; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const unsigned a = i < ntiles ? tcnt[2 * i] : 0u, b = i < ntiles ? tcnt[2 * i + 1] : 0u;
        unsigned ta, tb;
        const unsigned ea = block_excl_scan(a, sm, ta);
        const unsigned eb = block_excl_scan(b, sm, tb);
        if (i < ntiles) {
            tcnt[2 * i] = carry0 + ea;
            tcnt[2 * i + 1] = carry1 + eb;
        }
        carry0 += ta;
        carry1 += tb;
    }
    if (threadIdx.x == 0) {
        cnt[0] = carry0;
        cnt[1] = carry1;
    }
}
__global__ void __launch_bounds__(LT_THREADS) k_lists_write(int64_t n_nodes, const int8_t *__restrict__ nlev,
                                                            const uint8_t *__restrict__ nflag,
                                                            const int32_t *__restrict__ nbot,
                                                            const int32_t *__restrict__ ntop,
                                                            const uint32_t *__restrict__ tcnt, int32_t *leaf_list,
                                                            int32_t *p2m_list) {
    pdl_trigger();
    pdl_wait();
    __shared__ unsigned sm[32];
    unsigned oa = tcnt[2 * blockIdx.x], ob = tcnt[2 * blockIdx.x + 1];
    const int64_t g0 = (int64_t)blockIdx.x * LT_TILE;
    for (int k = 0; k < LT_TILE; k += LT_THREADS) {
        if (g0 + k >= n_nodes) break;  // uniform over the block
        const int64_t g = g0 + k + threadIdx.x;
        ListFlags f;
        if (g < n_nodes) f = list_flags(g, nlev, nflag, nbot, ntop);
        unsigned ta, tb;
        const unsigned ea = block_excl_scan(f.leaf, sm, ta);
        const unsigned eb = block_excl_scan(f.p2m, sm, tb);
        if (f.leaf) leaf_list[oa + ea] = (int32_t)g;
        if (f.p2m) p2m_list[ob + eb] = (int32_t)g;
        oa += ta;
        ob += tb;
    }
}

// Entries sorted by (level, key) with one block per level when every level
// fits in shared memory: block l picks the level-l entries out of the
// collected list, sorts them by the 2l key bits with an LSD radix sort in
// shared memory (8-bit digits; warp w ranks its contiguous chunk in order with
// warp_match_digit, so the sort is stable and the warps' chunks keep their
// order), and writes them at the level's offset (the counts of the levels
// above).  Keys are distinct within a level: a cell is either split or X-list.
constexpr int ES_THREADS = 1024, ES_WARPS = ES_THREADS / 32, ES_CAP = 12288;
// levels <= 10 rank through a bitmap of 4^10 bits (128 KB) plus 4096 group
// prefixes (16 KB), inside the radix sort's shared memory
constexpr int ES_BITMAP_LEVELS = 10;
constexpr size_t ES_SMEM = (size_t)2 * ES_CAP * sizeof(uint64_t) + (size_t)ES_WARPS * 256 * sizeof(uint32_t);
__global__ void __launch_bounds__(ES_THREADS) k_ent_sort(const uint64_t *__restrict__ list, int64_t n_ent,
                                                         const unsigned long long *__restrict__ lcount,
                                                         uint64_t *__restrict__ ent) {
    extern __shared__ __align__(16) unsigned char es_sm[];
    uint64_t *A = (uint64_t *)es_sm, *B = A + ES_CAP;
    uint32_t(*wcnt)[256] = (uint32_t(*)[256])(B + ES_CAP);
    __shared__ unsigned s_cnt, scan_sm[32];
    __shared__ long long s_eoff;
    pdl_trigger();
    pdl_wait();
    const int l = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int m = (int)lcount[l];
    if (m == 0 || (l > ES_BITMAP_LEVELS && m > ES_CAP)) return;  // the host sorts globally then
    if (threadIdx.x == 0) {
        long long o = 0;
        for (int q = 0; q < l; q++) o += (long long)lcount[q];
        s_eoff = o;
        s_cnt = 0;
    }
    __syncthreads();
    constexpr int U = 8;
    if (l <= ES_BITMAP_LEVELS) {
        // Levels up to ES_BITMAP_LEVELS have at most 4^l cells: one bit per
        // cell in shared memory, prefix counts over groups of 8 words, and an
        // entry's rank is the number of set bits below its key.
        uint32_t *bm = (uint32_t *)es_sm;                 // [4^l / 32] words
        uint32_t *gp = bm + (1u << (2 * ES_BITMAP_LEVELS - 5));  // group prefixes
        const int nwords = (int)(((1u << (2 * l)) + 31) >> 5), ngroups = (nwords + 7) >> 3;
        for (int i = threadIdx.x; i < nwords; i += ES_THREADS) bm[i] = 0;
        __syncthreads();
        for (int pass = 0; pass < 2; pass++) {
            for (int64_t base = 0; base < n_ent; base += (int64_t)U * ES_THREADS) {
                uint64_t e[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int64_t j = base + (int64_t)u * ES_THREADS + threadIdx.x;
                    e[u] = j < n_ent ? list[j] : ENT_EMPTY;
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (e[u] == ENT_EMPTY || (int)(e[u] >> ENT_LEVEL_SHIFT) != l) continue;
                    const uint32_t k = (uint32_t)((e[u] >> 1) & 0xFFFFFFFFull), wd = k >> 5, bit = k & 31;
                    if (pass == 0) {
                        atomicOr(&bm[wd], 1u << bit);
                    } else {
                        uint32_t r = gp[wd >> 3] + __popc(bm[wd] & ((1u << bit) - 1u));
                        for (uint32_t q = wd & ~7u; q < wd; q++) r += __popc(bm[q]);
                        ent[s_eoff + r] = e[u];
                    }
                }
            }
            if (pass == 0) {
                __syncthreads();
                // groups of 8 words: counts, then an exclusive scan (up to 4 groups per thread)
                const int per = (ngroups + ES_THREADS - 1) / ES_THREADS, g0 = threadIdx.x * per;
                uint32_t c[4] = {0, 0, 0, 0}, tsum = 0;
                for (int q = 0; q < per && q < 4; q++) {
                    const int g = g0 + q;
                    if (g < ngroups)
                        for (int i = 8 * g; i < 8 * g + 8 && i < nwords; i++) c[q] += __popc(bm[i]);
                    tsum += c[q];
                }
                unsigned total;
                unsigned run = block_excl_scan(tsum, scan_sm, total);
                for (int q = 0; q < per && q < 4; q++) {
                    const int g = g0 + q;
                    if (g < ngroups) gp[g] = run;
                    run += c[q];
                }
                __syncthreads();
            }
        }
        return;
    }
    for (int64_t base = 0; base < n_ent; base += (int64_t)U * ES_THREADS) {
        uint64_t e[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t j = base + (int64_t)u * ES_THREADS + threadIdx.x;
            e[u] = j < n_ent ? list[j] : ENT_EMPTY;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool mine = e[u] != ENT_EMPTY && (int)(e[u] >> ENT_LEVEL_SHIFT) == l;
            const unsigned bm = __ballot_sync(0xffffffffu, mine);
            if (!bm) continue;
            unsigned b0 = 0;
            if (lane == __ffs(bm) - 1) b0 = atomicAdd(&s_cnt, (unsigned)__popc(bm));
            b0 = __shfl_sync(0xffffffffu, b0, __ffs(bm) - 1);
            const unsigned pos = b0 + __popc(bm & ((1u << lane) - 1));
            if (mine && pos < ES_CAP) A[pos] = e[u];
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int chunk = ((m + ES_WARPS - 1) / ES_WARPS + 31) & ~31;
    const int c0 = min(w * chunk, m), c1 = min(c0 + chunk, m);
    for (int sh = 1; sh < 1 + 2 * l; sh += 8) {
        for (int d = lane; d < 256; d += 32) wcnt[w][d] = 0;
        __syncwarp();
        for (int i = c0 + lane; i - lane < c1; i += 32) {
            const bool ok = i < c1;
            const uint32_t d = ok ? (uint32_t)((A[i] >> sh) & 255) : 256u;
            const unsigned peers = warp_match_digit(d);
            if (ok && lane == __ffs(peers) - 1) wcnt[w][d] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint32_t tot = 0;
        if (threadIdx.x < 256) {
            for (int ww = 0; ww < ES_WARPS; ww++) {
                const uint32_t c = wcnt[ww][threadIdx.x];
                wcnt[ww][threadIdx.x] = tot;
                tot += c;
            }
        }
        unsigned total;
        const unsigned start = block_excl_scan(threadIdx.x < 256 ? tot : 0u, scan_sm, total);
        if (threadIdx.x < 256)
            for (int ww = 0; ww < ES_WARPS; ww++) wcnt[ww][threadIdx.x] += start;
        __syncthreads();
        for (int i = c0 + lane; i - lane < c1; i += 32) {
            const bool ok = i < c1;
            const uint64_t k = ok ? A[i] : 0;
            const uint32_t d = ok ? (uint32_t)((k >> sh) & 255) : 256u;
            const unsigned peers = warp_match_digit(d);
            if (ok) {
                const uint32_t b = wcnt[w][d];
                B[b + __popc(peers & lt)] = k;
            }
            __syncwarp();
            if (ok && lane == __ffs(peers) - 1) wcnt[w][d] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint64_t *t = A;
        A = B;
        B = t;
    }
    const long long eoff = s_eoff;
    for (int i = threadIdx.x; i < m; i += ES_THREADS) ent[eoff + i] = A[i];
}

// Work counts: cnt[0] P2P pairs, cnt[1] P2M points, cnt[2] V-list pairs,
// cnt[3] (target group, direction) M2L blocks.  The V-list pairs are those of
// kifmm_export_lists: targets the children of split cells, sources the
// children of a colleague's non-empty child group, well separated.
__global__ void k_stats(LevelTable T, const uint64_t *__restrict__ ent, const int32_t *__restrict__ ent_node,
                        const int32_t *__restrict__ leaf_list, int64_t nleaf, const int32_t *__restrict__ p2m_list,
                        int64_t np2m, const int32_t *__restrict__ nbot, const int32_t *__restrict__ ntop,
                        const int32_t *__restrict__ ncoll, const int32_t *__restrict__ nent, int64_t n_ent,
                        unsigned long long *cnt) {
    int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long a = 0, b = 0, c = 0, d = 0;
    for (int64_t i = tid; i < nleaf; i += stride) {
        int g = leaf_list[i];
        int64_t s = 0;
        for (int k = 0; k < 9; k++) {
            int q = ncoll[9 * (int64_t)g + k];
            if (q >= 0) s += ntop[q] - nbot[q];
        }
        a += (unsigned long long)((ntop[g] - nbot[g]) * s);
    }
    for (int64_t i = tid; i < np2m; i += stride) b += ntop[p2m_list[i]] - nbot[p2m_list[i]];
    for (int64_t j = tid; j < n_ent; j += stride) {
        if (ent[j] & 1) continue;
        int l = (int)(ent[j] >> ENT_LEVEL_SHIFT);
        if (l < 1) continue;
        int p = ent_node[j];
        for (int dd = 0; dd < 9; dd++) {
            if (dd == 4) continue;
            if (m2l_source_entry(ncoll, nent, nbot, ntop, p, dd) < 0) continue;
            d++;
            int dx = dd / 3 - 1, dy = dd % 3 - 1;
            for (int ta = 0; ta < 4; ta++)
                for (int sb = 0; sb < 4; sb++) {
                    int ox = 2 * dx - (ta >> 1) + (sb >> 1), oy = 2 * dy - (ta & 1) + (sb & 1);
                    if (ox < -1 || ox > 1 || oy < -1 || oy > 1) c++;
                }
        }
    }
    atomicAdd(&cnt[0], a); atomicAdd(&cnt[1], b); atomicAdd(&cnt[2], c); atomicAdd(&cnt[3], d);
}

// Morton keys of n points on the root box [m, M] (k_keys), launch only.
void launch_morton_keys(const double *x, const double *y, int64_t n, double m, double M, uint64_t *key,
                        int32_t *perm, unsigned long long *outside, int num_sms, cudaStream_t stream) {
    double h = M > m ? std::ldexp(M - m, -KEY_DEPTH) : 0.0;
    k_keys<<<grid_for(n, 256, num_sms * 8), 256, 0, stream>>>(x, y, n, m, M, h, key, perm, outside);
    KIFMM_LAUNCHED();
}

struct FillArgs {
    uint32_t *p[6];
    size_t n[6];
    uint32_t v[6];
    int k;
};
__global__ void k_fill(FillArgs F) {
    pdl_trigger();
    pdl_wait();  // the previous kernel may still read what is overwritten here
    const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, ts = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < F.k; r++) {
        uint32_t *p = F.p[r];
        const size_t n = F.n[r];
        const uint32_t v = F.v[r];
        size_t head = 0;  // words before the first 16-byte boundary
        while (head < n && (((uintptr_t)(p + head)) & 15)) head++;
        for (size_t i = t0; i < head; i += ts) p[i] = v;
        uint4 *q = (uint4 *)(p + head);
        const size_t nq = (n - head) / 4;
        for (size_t i = t0; i < nq; i += ts) q[i] = make_uint4(v, v, v, v);
        for (size_t i = head + 4 * nq + t0; i < n; i += ts) p[i] = v;
    }
}

void launch_fill(kifmm_plan *P, std::initializer_list<FillRange> ranges) {
    FillArgs F{};
    size_t words = 0;
    for (const FillRange &r : ranges) {
        KIFMM_REQUIRE(F.k < 6, KIFMM_ERR_ARG, "launch_fill: at most six ranges");
        if (!r.words) continue;
        F.p[F.k] = (uint32_t *)r.p;
        F.n[F.k] = r.words;
        F.v[F.k] = r.value;
        F.k++;
        words += r.words;
    }
    if (!F.k) return;
    const unsigned grid = grid_for((int64_t)((words + 3) / 4), 256, P->num_sms * 8);
    launch_pdl(k_fill, dim3(grid), dim3(256), 0, P->stream, F);
}

static void build_tree_impl(kifmm_plan *P, const double *x, const double *y, int64_t n, int mem) {
    KIFMM_REQUIRE(n > 0 && n < (1ll << 31) - 1, KIFMM_ERR_ARG, "build_tree: need 0 < n < 2^31-1 points");
    KIFMM_REQUIRE(x && y, KIFMM_ERR_ARG, "build_tree: null coordinate pointer");
    cudaStream_t s = P->stream;
    P->have_tree = P->have_ops = P->have_expansions = false;
    P->N = n;
    // The coordinates are read only inside this call (root box, keys, the
    // gather into Morton order, all complete before it returns): device
    // arrays are read in place, host arrays are uploaded once.
    const double *xd = x, *yd = y;
    if (mem != KIFMM_MEM_DEVICE) {
        P->x.alloc(n); P->y.alloc(n);
        KIFMM_CUDA(cudaMemcpyAsync(P->x.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
        KIFMM_CUDA(cudaMemcpyAsync(P->y.p, y, n * sizeof(double), cudaMemcpyHostToDevice, s));
        xd = P->x.p;
        yd = P->y.p;
    }
    P->scal.alloc(KIFMM_SCAL_WORDS);
    KIFMM_CUDA(cudaMemcpyAsync(P->scal.p, P->hpin + HP_INIT, 16 * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                               s));
    const int TB = 256;
    unsigned gs = grid_for(n, TB, P->num_sms * 8);
    k_bbox<<<gs, TB, 0, s>>>(xd, yd, n, P->scal.p);
    KIFMM_LAUNCHED();
    P->pkey.alloc(n); P->perm.alloc(n); P->key2.alloc(n); P->perm2.alloc(n);
    // the root box stays on the device until the counts below come back
    launch_pdl(k_keys_dev, dim3(gs), dim3(TB), 0, s, xd, yd, n,
               (int)P->opt.fix_bbox, (const unsigned long long *)P->scal.p, P->pkey.p, P->perm.p, P->scal.p + 8);
    // Sort by the top 32 key bits first (levels 1..16, four 8-bit passes): that
    // orders every cell of level <= 16, enough whenever no split lies deeper
    // than level 15.  Otherwise sort all 58 bits and count again.
    constexpr int FAST_BITS = 32, FAST_LEVELS = FAST_BITS / 2;
    {
        PhaseScope ph(P, KIFMM_PHASE_SORT);
        radix_sort_pairs_bits(P->pkey.p, P->perm.p, P->key2.p, P->perm2.p, n, 2 * KEY_DEPTH - FAST_BITS, FAST_BITS, P);
    }
    HashSet H{};
    H.count = P->scal.p + 9;
    H.ovf = P->scal.p + 10;
    P->misc.alloc(128);
    P->m2l_hist.alloc((size_t)(MAX_LEVELS + 1) * M2L_KEYS);
    unsigned long long *lc = (unsigned long long *)P->misc.p;  // [32] entries per level
    unsigned long long lcount[32] = {};
    const unsigned cgrid = grid_for((n + 31) / 32 * 32, TB, P->num_sms * 64);
    ensure_side(P);
    // The split-cell set for a list capacity: table and list sized and
    // cleared, the closure and the X-list, then count, overflow and per-level
    // counts to the host, marked by tree_ev.
    bool misc_cleared = false;  // by a queued split-cell set (launch_fill below)
    auto queue_closure = [&](uint64_t cap) {
        misc_cleared = true;
        uint64_t hcap = 1;
        while (hcap < 2 * cap) hcap <<= 1;
        P->hash.alloc(hcap);
        P->hash_cap = hcap;
        P->list.alloc(cap);
        // one launch clears the table (all ones), the set's count and overflow
        // flag, the per-level entry counts and the later list counters (misc),
        // and the M2L target order's histogram
        launch_fill(P, {{P->hash.p, 2 * hcap, 0xFFFFFFFFu},
                        {P->scal.p + 9, 4, 0u},
                        {P->misc.p, 2 * 128, 0u},
                        {P->m2l_hist.p, (size_t)(MAX_LEVELS + 1) * M2L_KEYS, 0u}});
        H.tab = (unsigned long long *)P->hash.p;
        H.mask = hcap - 1;
        H.list = P->list.p;
        H.cap = cap;
        H.lcount = lc;
        launch_pdl(k_closure, dim3(cgrid), dim3(TB), 0, s, (const uint64_t *)P->pkey.p, n, (int64_t)P->ppl, H);
        // the X-list reads the complete split set: nine items per entry, grid-stride
        launch_pdl(k_xlist, dim3(grid_for(9 * (int64_t)cap, TB, P->num_sms * 8)), dim3(TB), 0, s, H);
        KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_SCAL + 9, P->scal.p + 9, 2 * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, s));
        KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_MISC, lc, sizeof(lcount), cudaMemcpyDeviceToHost, s));
        KIFMM_CUDA(cudaEventRecord(P->tree_ev, s));
    };
    unsigned long long sc[9];  // [0..3] ordered extremes, [4] non-finite, [5..7] T0 count/depth/overflow, [8] outside
    unsigned long long *st = sc + 5;
    // T0 counts and the root box go to the host (marked by ops_fork, after
    // which the operators may start); the split-cell set is queued right
    // behind them, before the counts are seen, with the capacity of the last
    // build (or an estimate from n): it is kept if the sort by the top 32 key
    // bits was enough and the set fitted, and rebuilt otherwise.
    bool spec = n > P->ppl;
    uint64_t spec_cap = P->spec_cap;
    if (!spec_cap)
        spec_cap = std::min<uint64_t>(16 * (uint64_t)std::max<int64_t>(n / P->ppl, 1), 2 * (uint64_t)n) + 4096;
    for (int full = 0; full < 2; full++) {
        // T0 count, depth and overflow: still zero from the reset copy at the
        // start of this call on the first pass
        if (full) KIFMM_CUDA(cudaMemsetAsync(P->scal.p + 5, 0, 3 * sizeof(unsigned long long), s));
        launch_pdl(k_t0_count, dim3(gs), dim3(TB), 0, s, (const uint64_t *)P->pkey.p, n, (int64_t)P->ppl, P->scal.p);
        KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_SCAL, P->scal.p, sizeof(sc), cudaMemcpyDeviceToHost, s));
        KIFMM_CUDA(cudaEventRecord(P->ops_fork, s));
        if (spec && full == 0) {
            PhaseScope ph_c(P, KIFMM_PHASE_CLOSURE);
            queue_closure(spec_cap);
        }
        KIFMM_CUDA(cudaEventSynchronize(P->ops_fork));
        memcpy(sc, P->hpin + HP_SCAL, sizeof(sc));
        if (full == 0) {
            KIFMM_REQUIRE(sc[4] == 0, KIFMM_ERR_ARG, "build_tree: non-finite coordinates");
            double m, M;
            root_box(sc, P->opt.fix_bbox, m, M);
            KIFMM_REQUIRE(std::fabs(m) < 8388608.0 && std::fabs(M) < 8388608.0, KIFMM_ERR_RANGE,
                          "build_tree: |coordinates| must stay below 2^23 for exact dyadic midpoints");
            P->root_min = m; P->root_max = M; P->W = M - m;
            KIFMM_REQUIRE(P->W > 0 || n <= P->ppl, KIFMM_ERR_DEPTH,
                          "build_tree: more than Ncutoff points on one integer point (zero-width root box)");
        }
        if (full || (st[1] <= (unsigned long long)FAST_LEVELS && st[2] == 0)) break;
        spec = false;  // the queued set used the partial order: rebuilt below
        PhaseScope ph(P, KIFMM_PHASE_SORT);
        radix_sort_pairs(P->pkey.p, P->perm.p, P->key2.p, P->perm2.p, n, 2 * KEY_DEPTH, P);
    }
    P->xs.alloc(n); P->ys.alloc(n);
    launch_pdl(k_gather2, dim3(gs), dim3(TB), 0, s, xd, yd,
               (const int32_t *)P->perm.p, n, P->xs.p, P->ys.p);
    P->n_outside = (int64_t)st[3];
    KIFMM_REQUIRE(st[2] == 0, KIFMM_ERR_DEPTH,
                  "build_tree: more than Ncutoff points share one cell of the finest grid (2^29 per side); "
                  "the tree would need more than 30 levels");
    int L = n > P->ppl ? (int)st[1] + 1 : 1;
    KIFMM_REQUIRE(L <= MAX_LEVELS, KIFMM_ERR_DEPTH, "build_tree: too many levels");
    P->L = L;
    const uint64_t t0count = st[0];
    // the operators need only the root width and the depth: they run on the
    // side stream while the split-cell set and the node tables are built
    start_operators(P, true);

    int64_t n_ent = 0;
    if (L > 1) {
        PhaseScope ph_c(P, KIFMM_PHASE_CLOSURE);
        const uint64_t exact = t0count * 16 + 4096;
        for (int attempt = 0;; attempt++) {
            uint64_t cap = spec_cap;
            if (!spec || attempt > 0) {
                cap = exact << (2 * std::max(attempt - (spec ? 1 : 0), 0));
                queue_closure(cap);
            }
            KIFMM_CUDA(cudaEventSynchronize(P->tree_ev));
            unsigned long long cv[2];
            memcpy(cv, P->hpin + HP_SCAL + 9, sizeof(cv));
            memcpy(lcount, P->hpin + HP_MISC, sizeof(lcount));
            if (cv[1] == 0 && cv[0] <= cap) {
                n_ent = (int64_t)cv[0];
                break;
            }
            KIFMM_REQUIRE(attempt < 5, KIFMM_ERR_NOMEM, "build_tree: split-cell set overflow");
        }
        P->spec_cap = exact;
    }
    P->n_ent = n_ent;
    P->ent.alloc(n_ent);
    P->key2.alloc(std::max<int64_t>(n, n_ent));
    if (n_ent) {
        PhaseScope ph_e(P, KIFMM_PHASE_ENTRIES);
        unsigned long long lmax = 0;  // the largest level that k_ent_sort radix-sorts
        for (int l = ES_BITMAP_LEVELS + 1; l < L; l++) lmax = std::max(lmax, lcount[l]);
        if (lmax <= (unsigned long long)ES_CAP) {
            ensure_dyn_smem(k_ent_sort, ES_SMEM);
            launch_pdl(k_ent_sort, dim3((unsigned)L), dim3(ES_THREADS), ES_SMEM, s, (const uint64_t *)P->list.p,
                       n_ent, (const unsigned long long *)lc, P->ent.p);
        } else {
            KIFMM_CUDA(cudaMemcpyAsync(P->ent.p, P->list.p, n_ent * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
            // entry = (level << 57) | (key << 1) | xlist with keys of at most 2(L-1)
            // bits: sort the digits holding key bits, then the level digit
            int shifts[8], np = 0;
            for (int sh = 0; sh <= 2 * (L - 1); sh += 8) shifts[np++] = sh;
            if (8 * np > 56) {
                np = 0;
                for (int sh = 0; sh < 64; sh += 8) shifts[np++] = sh;
            } else {
                shifts[np++] = 56;
            }
            radix_sort_keys_shifts(P->ent.p, P->key2.p, n_ent, shifts, np, P);
        }
    }
    // per-level entry counts (counted as the entries were added) -> level table
    LevelTable &T = P->lt;
    memset(&T, 0, sizeof(T));
    T.L = L;
    int64_t off = 0, eoff = 0;
    for (int l = 0; l < L; l++) {
        int64_t nl = l == 0 ? 1 : 4 * (int64_t)lcount[l - 1];
        T.off[l] = off; T.eoff[l] = eoff; T.ne[l] = (int64_t)lcount[l];
        P->lv[l].off = off; P->lv[l].n = nl; P->lv[l].eoff = eoff; P->lv[l].ne = (int64_t)lcount[l];
        P->lv[l].width = std::ldexp(P->W, -l);
        off += nl;
        eoff += (int64_t)lcount[l];
    }
    T.off[L] = off; T.eoff[L] = eoff;
    KIFMM_REQUIRE(lcount[L - 1] == 0 && eoff == n_ent, KIFMM_ERR_CUDA, "build_tree: inconsistent level table");
    int64_t NN = off;
    KIFMM_REQUIRE(NN < (1ll << 31), KIFMM_ERR_ARG, "build_tree: too many nodes");
    P->n_nodes = NN;
    std::optional<PhaseScope> ph_n;
    ph_n.emplace(P, KIFMM_PHASE_NODES);
    P->nkey.alloc(NN); P->nlev.alloc(NN); P->nflag.alloc(NN); P->nbot.alloc(NN); P->ntop.alloc(NN);
    P->nparent.alloc(NN); P->nchild.alloc(NN); P->nent.alloc(NN); P->ncoll.alloc(9 * NN);
    P->ent_node.alloc(std::max<int64_t>(n_ent, 1));
    P->leaf_list.alloc(NN); P->p2m_list.alloc(NN);
    unsigned ng = grid_for(NN, TB, P->num_sms * 16);
    EntryIndex X{(const unsigned long long *)P->hash.p, nullptr, (uint64_t)(P->hash_cap - 1)};
    if (n_ent) {
        P->hash_idx.alloc(P->hash_cap);
        X.hidx = P->hash_idx.p;
        launch_pdl(k_hash_index, dim3(grid_for(n_ent, TB, P->num_sms * 8)), dim3(TB), 0, s, (const uint64_t *)P->ent.p,
                   (int64_t)n_ent, X.tab, X.mask, P->hash_idx.p);
    }
    launch_pdl(k_nodes, dim3(ng), dim3(TB), 0, s, T, X, NN, P->ent.p, P->pkey.p, n, P->nkey.p, P->nlev.p, P->nflag.p, P->nbot.p, P->ntop.p,
                              P->nparent.p, P->nchild.p, P->nent.p, P->ncoll.p, P->ent_node.p);
    KIFMM_LAUNCHED();
    unsigned long long *cnt = (unsigned long long *)P->misc.p + 32;
    unsigned long long *lcnt = (unsigned long long *)P->misc.p + 64;  // [MAX_LEVELS] leaves per level
    // cnt and lcnt were cleared with the split-cell set (launch_fill above);
    // a single-leaf tree queued none
    if (!misc_cleared) launch_fill(P, {{P->misc.p, 2 * 128, 0u}});
    {
        const int64_t ntiles = (NN + LT_TILE - 1) / LT_TILE;
        P->list_tiles.alloc(2 * ntiles);
        launch_pdl(k_lists_count, dim3((unsigned)ntiles), dim3(LT_THREADS), 0, s, NN, P->nlev.p, P->nflag.p, P->nbot.p, P->ntop.p,
                                                              P->list_tiles.p, cnt, lcnt);
        KIFMM_LAUNCHED();
        launch_pdl(k_lists_scan, dim3(1), dim3(1024), 0, s, ntiles, P->list_tiles.p, cnt);
        KIFMM_LAUNCHED();
        launch_pdl(k_lists_write, dim3((unsigned)ntiles), dim3(LT_THREADS), 0, s, NN, P->nlev.p, P->nflag.p, P->nbot.p, P->ntop.p,
                                                              P->list_tiles.p, P->leaf_list.p, P->p2m_list.p);
        KIFMM_LAUNCHED();
    }
    unsigned long long c5[5], sort_err = 0, lv[MAX_LEVELS];
    // misc[32..128) holds cnt (at 32) and lcnt (at 64)
    static_assert(64 + MAX_LEVELS <= 128, "misc layout");
    KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_MISC + 32, cnt, 96 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_SCAL + KIFMM_SCAL_SORT_ERR, P->scal.p + KIFMM_SCAL_SORT_ERR,
                               sizeof(sort_err), cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaEventRecord(P->tree_ev, s));
    // the M2L target order needs only the entries and the node tables: it runs
    // while the host waits for the counts
    build_m2l_order(P);
    KIFMM_CUDA(cudaEventSynchronize(P->tree_ev));
    memcpy(c5, P->hpin + HP_MISC + 32, sizeof(c5));
    memcpy(lv, P->hpin + HP_MISC + 64, sizeof(lv));
    sort_err = P->hpin[HP_SCAL + KIFMM_SCAL_SORT_ERR];
    KIFMM_REQUIRE(sort_err == 0, KIFMM_ERR_CUDA, "build_tree: a radix-sort look-back wait timed out");
    P->n_leaf_list = (int64_t)c5[0];
    P->leaf_loff[0] = 0;
    for (int l = 0; l < MAX_LEVELS; l++) P->leaf_loff[l + 1] = P->leaf_loff[l] + (int64_t)lv[l];
    KIFMM_REQUIRE(P->leaf_loff[MAX_LEVELS] == P->n_leaf_list, KIFMM_ERR_CUDA, "build_tree: inconsistent leaf counts");
    P->n_p2m_list = (int64_t)c5[1];
    ph_n.reset();
    P->n_leaves = (int64_t)c5[2];
    P->n_fake = (int64_t)c5[3];
    P->n_xlist = (int64_t)c5[4];
    P->have_stats = false;
    build_leaf_records(P);
    P->have_tree = true;
}

void build_tree(kifmm_plan *P, const double *x, const double *y, int64_t n, int mem) {
    try {
        build_tree_impl(P, x, y, n, mem);
    } catch (...) {
        // device coordinates are read in place: nothing may still read them
        // once the call has returned, error or not
        cudaStreamSynchronize(P->stream);
        throw;
    }
}

// Work counts for reporting (kifmm_get_tree_info), computed on request.
void tree_stats(kifmm_plan *P) {
    if (P->have_stats) return;
    cudaStream_t s = P->stream;
    unsigned long long *cnt = (unsigned long long *)P->misc.p + 40;
    KIFMM_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned long long), s));
    k_stats<<<P->num_sms * 2, 256, 0, s>>>(P->lt, P->ent.p, P->ent_node.p, P->leaf_list.p, P->n_leaf_list,
                                             P->p2m_list.p, P->n_p2m_list, P->nbot.p, P->ntop.p, P->ncoll.p,
                                             P->nent.p, P->n_ent, cnt);
    KIFMM_LAUNCHED();
    unsigned long long c4[4];
    KIFMM_CUDA(cudaMemcpyAsync(P->hpin + HP_STATS, cnt, sizeof(c4), cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaStreamSynchronize(s));
    memcpy(c4, P->hpin + HP_STATS, sizeof(c4));
    P->n_p2p_pairs = (int64_t)c4[0];
    P->n_p2m_points = (int64_t)c4[1];
    P->n_m2l_pairs = (int64_t)c4[2];
    P->n_m2l_groups = (int64_t)c4[3];
    P->have_stats = true;
}

void export_tree(kifmm_plan *P, int64_t *nodes, int64_t *point_leaf) {
    KIFMM_REQUIRE(P->have_tree, KIFMM_ERR_STATE, "export_tree: no tree");
    int64_t NN = P->n_nodes, n = P->N;
    std::vector<uint64_t> key(NN);
    std::vector<int8_t> lev(NN);
    std::vector<uint8_t> fl(NN);
    std::vector<int32_t> bot(NN), top(NN), perm(n);
    cudaStream_t s = P->stream;
    KIFMM_CUDA(cudaMemcpyAsync(key.data(), P->nkey.p, NN * 8, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(lev.data(), P->nlev.p, NN, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(fl.data(), P->nflag.p, NN, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(bot.data(), P->nbot.p, NN * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(top.data(), P->ntop.p, NN * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(perm.data(), P->perm.p, n * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaStreamSynchronize(s));
    for (int64_t g = 0; g < NN; g++) {
        uint64_t k = key[g];
        int64_t ix = (int64_t)compact2(k >> 1), iy = (int64_t)compact2(k);
        bool fake = fl[g] & NF_FAKE, split = fl[g] & NF_SPLIT, xl = fl[g] & NF_XLIST;
        bool leaf = !fake && !split;
        if (nodes) {
            int64_t *r = nodes + 7 * g;
            r[0] = lev[g]; r[1] = ix; r[2] = iy; r[3] = leaf; r[4] = fake; r[5] = xl; r[6] = top[g] - bot[g];
        }
        if (point_leaf && leaf)
            for (int32_t p = bot[g]; p < top[g]; p++) {
                int64_t *q = point_leaf + 3 * (int64_t)perm[p];
                q[0] = lev[g]; q[1] = ix; q[2] = iy;
            }
    }
}

// Interaction lists as the apply kernels walk them (kifmm_export_lists):
// colleagues from the node table; M2L pairs from the split entries of levels
// 1..L-2 and m2l_source_entry (the test k_m2l_d, k_m2l_f and k_m2l_tc make);
// P2P pairs from the leaf list and its colleagues with points (the leaf
// kernels).  Node numbers are kifmm_export_tree's rows.
void export_lists(kifmm_plan *P, int64_t *coll, int64_t *m2l, int64_t *n_m2l, int64_t *p2p, int64_t *n_p2p) {
    KIFMM_REQUIRE(P->have_tree, KIFMM_ERR_STATE, "export_lists: no tree");
    const int64_t NN = P->n_nodes, NE = P->n_ent, NL = P->n_leaf_list;
    std::vector<int32_t> cl(9 * NN), bot(NN), top(NN), nent(NN), en(NE), leaves(NL);
    std::vector<uint64_t> ent(NE);
    cudaStream_t s = P->stream;
    KIFMM_CUDA(cudaMemcpyAsync(cl.data(), P->ncoll.p, 9 * NN * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(bot.data(), P->nbot.p, NN * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(top.data(), P->ntop.p, NN * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaMemcpyAsync(nent.data(), P->nent.p, NN * 4, cudaMemcpyDeviceToHost, s));
    if (NE) {
        KIFMM_CUDA(cudaMemcpyAsync(ent.data(), P->ent.p, NE * 8, cudaMemcpyDeviceToHost, s));
        KIFMM_CUDA(cudaMemcpyAsync(en.data(), P->ent_node.p, NE * 4, cudaMemcpyDeviceToHost, s));
    }
    if (NL) KIFMM_CUDA(cudaMemcpyAsync(leaves.data(), P->leaf_list.p, NL * 4, cudaMemcpyDeviceToHost, s));
    KIFMM_CUDA(cudaStreamSynchronize(s));
    if (coll)
        for (int64_t i = 0; i < 9 * NN; i++) coll[i] = cl[i];
    int64_t nm = 0, cap_m = (m2l && n_m2l) ? *n_m2l : 0;
    for (int64_t j = 0; j < NE; j++) {
        if (ent[j] & 1) continue;  // X-list cell: its fake children receive no M2L
        const int l = (int)(ent[j] >> ENT_LEVEL_SHIFT);
        if (l < 1 || l > P->L - 2) continue;
        const int p = en[j];
        const int64_t t0 = P->lt.off[l + 1] + 4 * (j - P->lt.eoff[l]);
        for (int dd = 0; dd < 9; dd++) {
            if (dd == 4) continue;
            const int je = m2l_source_entry(cl.data(), nent.data(), bot.data(), top.data(), p, dd);
            if (je < 0) continue;
            const int64_t s0 = P->lt.off[l + 1] + 4 * (je - P->lt.eoff[l]);
            const int dx = dd / 3 - 1, dy = dd % 3 - 1;
            for (int ta = 0; ta < 4; ta++)
                for (int sb = 0; sb < 4; sb++) {
                    const int ox = 2 * dx - (ta >> 1) + (sb >> 1), oy = 2 * dy - (ta & 1) + (sb & 1);
                    if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1) continue;
                    if (m2l) {
                        KIFMM_REQUIRE(nm < cap_m, KIFMM_ERR_ARG, "export_lists: m2l buffer smaller than *n_m2l pairs");
                        m2l[2 * nm] = t0 + ta;
                        m2l[2 * nm + 1] = s0 + sb;
                    }
                    nm++;
                }
        }
    }
    int64_t np = 0, cap_p = (p2p && n_p2p) ? *n_p2p : 0;
    for (int64_t i = 0; i < NL; i++) {
        const int g = leaves[i];
        for (int dd = 0; dd < 9; dd++) {
            const int c = cl[9 * (int64_t)g + dd];
            if (c < 0 || top[c] <= bot[c]) continue;
            if (p2p) {
                KIFMM_REQUIRE(np < cap_p, KIFMM_ERR_ARG, "export_lists: p2p buffer smaller than *n_p2p pairs");
                p2p[2 * np] = g;
                p2p[2 * np + 1] = c;
            }
            np++;
        }
    }
    if (n_m2l) *n_m2l = nm;
    if (n_p2p) *n_p2p = np;
}

}  // namespace kifmm
