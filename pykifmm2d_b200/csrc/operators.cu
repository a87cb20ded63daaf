// operators.cu -- per-level translation operators, built in FP64 on the GPU.
//
// Reference: FMM.precompute (pykifmm2d/class_fmm.py:182-298).
//   equivalent circle r1 = (sqrt2 + 0.01) w/2, check circle r2 = (4 - sqrt2 - 0.02) w/2,
//   Q points at theta_q = 2 pi q / Q (get_level_information, :35-45, :192);
//   E2C_l = G(small -> large)  (:213-217, LU-factored there; inverted here);
//   M2MC_l = G(children's small circles -> parent's large circle)  (:219-235);
//   M2LS_l[o] = G(small + o w -> small), o in [-3,3]^2 minus the 3x3 block (:237-250);
//   CM2LS_l[d] = the 4Q x 4Q child-to-child blocks for parent direction d (:252-285).
// The passes keep check potentials (u) rather than equivalent densities, so
// the inverse is composed into every operator:
//   M2M:  u_up(parent)   = sum_q (M2MC_l[:, q] Inv_{l+1}) u_up(child q)
//   L2L:  u_down(child q) = (M2MC_l[:, q])^T Inv_l u_down(parent)
//   M2L:  u_down(children of p) += (CM2LS_l[d] blockdiag(Inv_l)) u_up(children of p + d)
//   L2P:  equivalent density Inv_l u_down, evaluated on the check circle.
// Operators are stored column-major (element (r, c) at c * rows + r) so that
// threads owning consecutive rows read consecutive addresses.
#include <cmath>

#include "kifmm_internal.cuh"

namespace kifmm {

struct OpsArgs {
    int L, Q, kind;         // Q: state length per node (2 Nequiv for a complex kernel)
    int Qc, cplx;           // points per circle; complex kernel (realified operators)
    int circulant;          // E2C inverse from the DFT of its first row (KIFMM_E2C_CIRCULANT)
    double k;
    double W;
    double rf1, rf2;
    size_t stride;          // doubles per level block
    double *ops;            // level blocks
    double *poff;           // temp [L][49][Q][Q] = M2LS . Inv (row-major)
};

// level block layout (offsets in doubles)
__host__ __device__ inline size_t off_inv(int) { return 0; }
__host__ __device__ inline size_t off_m2m(int Q) { return (size_t)Q * Q; }
__host__ __device__ inline size_t off_l2l(int Q) { return (size_t)5 * Q * Q; }
__host__ __device__ inline size_t off_m2l(int Q) { return (size_t)9 * Q * Q; }
__host__ __device__ inline size_t off_large(int Q) { return (size_t)153 * Q * Q; }
__host__ __device__ inline size_t off_small(int Q) { return (size_t)153 * Q * Q + 2 * Q; }
__host__ __device__ inline size_t ops_stride(int Q) { return ((size_t)153 * Q * Q + 4 * Q + 31) & ~(size_t)31; }

__device__ __forceinline__ double lvl_width(const OpsArgs &A, int l) { return ldexp(A.W, -l); }

__device__ __forceinline__ double gval(const OpsArgs &A, double sx, double sy, double tx, double ty) {
    double dx = tx - sx, dy = ty - sy;
    return green_d(A.kind, A.k, dx * dx + dy * dy);
}
// Entry (rt, cs) of a kernel matrix on the state index space: source point cs
// of (sx, sy) shifted by (ox, oy), target point rt of (tx, ty).  Real values:
// G itself.  Complex values act on states [Re (Qc), Im (Qc)], so the matrix
// is the real image of the complex one: block (bt, bs) of entry
// (rt mod Qc, cs mod Qc) is Re G, -Im G (bt 0, bs 1), Im G (bt 1, bs 0), Re G.
// The real image of a transpose is not the transpose of the real image (that
// is the image of the conjugate transpose): with `tr` the entry is that of
// the image of the transposed matrix at (cs, rt), i.e. the blocks swap roles.
__device__ __forceinline__ double gent(const OpsArgs &A, const double *sx, const double *sy, double ox, double oy,
                                       const double *tx, const double *ty, int rt, int cs, bool tr = false) {
    if (!A.cplx) return gval(A, sx[cs] + ox, sy[cs] + oy, tx[rt], ty[rt]);
    const int pr = rt % A.Qc, ps = cs % A.Qc;
    const int bt = (tr ? cs : rt) / A.Qc, bs = (tr ? rt : cs) / A.Qc;
    const double dx = tx[pr] - (sx[ps] + ox), dy = ty[pr] - (sy[ps] + oy);
    const double2 g = green_z(A.kind, A.k, dx * dx + dy * dy);
    return bt == bs ? g.x : (bt == 0 ? -g.y : g.y);
}

// Gauss-Jordan with partial pivoting on [E2C | I], one warp per level: lane r
// owns row r of the augmented matrix (rows of 2Q+1 doubles in shared memory,
// conflict-free), so a pivot step needs warp synchronisation only.  Rows
// beyond 32 are taken by the same lanes in turn.  Per element the arithmetic
// is the block-wide form's: a[k][c] /= pivot, a[r][c] -= a[r][k] * a[k][c].
// One block per level: the circles, then the inverse of the Q x Q
// equivalent-to-check matrix by Gauss-Jordan elimination with partial
// pivoting on [E | I] (Q x 2Q), shared over the block: warp 0 picks the pivot,
// then every thread produces its elements of the next matrix from the current
// one (two buffers, so a step needs no separate read and write phases).
constexpr int INV_THREADS = 256;
static_assert(INV_THREADS % 128 == 0, "the elimination maps 128 columns (2 Nequiv <= 128) per row phase");
__global__ void __launch_bounds__(INV_THREADS) k_ops_inverse(OpsArgs A) {
    extern __shared__ double sm[];
    __shared__ int s_piv;
    const int Q = A.Q, Q2 = 2 * Q, ld = Q2 + 1, l = blockIdx.x, tid = threadIdx.x;
    if (l >= A.L) return;
    {  // the level's circles (get_level_information, class_fmm.py:35-45)
        const double w = lvl_width(A, l), r1 = 0.5 * w * A.rf1, r2 = 0.5 * w * A.rf2;
        double *bw = A.ops + (size_t)l * A.stride;
        const int Qc = A.Qc;  // circle points: x at [0, Qc), y at [Qc, 2 Qc)
        for (int q = tid; q < Qc; q += INV_THREADS) {
            const double th = q * (2.0 * 3.141592653589793 / Qc);
            const double c = cos(th), s = sin(th);
            bw[off_large(Q) + q] = r2 * c;
            bw[off_large(Q) + Qc + q] = r2 * s;
            bw[off_small(Q) + q] = r1 * c;
            bw[off_small(Q) + Qc + q] = r1 * s;
        }
        __syncthreads();
    }
    if (l < 1) return;
    double *a = sm, *nb = sm + (size_t)Q * ld;  // current and next matrix, Q x ld each
    const double *b = A.ops + (size_t)l * A.stride;
    const double *lx = b + off_large(Q), *ly = lx + A.Qc, *sx = b + off_small(Q), *sy = sx + A.Qc;
    if (A.circulant) {
        // E2C[t][s] = G(small_s -> large_t) depends on (s - t) mod Q only (both
        // circles carry the same Q angles and G is radial): E2C = C(a) with
        // a_j = G(small_j -> large_0), and C(a) C(b) = C(a (*) b) (circular
        // convolution), so the inverse is C(b) with DFT(b) = 1 / DFT(a).  a is
        // even (a_j = a_{Q-j}), so DFT(a) is real: lambda_m = sum_j a_j
        // cos(2 pi j m / Q), b_j = (1/Q) sum_m cos(2 pi j m / Q) / lambda_m.
        // The reference solves with the same diagonalisation by the FFT
        // (svd_fmm.py:239-242, :281-290); at Q <= 64 the DFT is formed directly.
        double *av = sm, *lam = sm + Q, *bv = sm + 2 * Q;
        for (int j = tid; j < Q; j += INV_THREADS) av[j] = gval(A, sx[j], sy[j], lx[0], ly[0]);
        __syncthreads();
        for (int m = tid; m < Q; m += INV_THREADS) {
            double acc = 0.0;
            for (int j = 0; j < Q; j++) acc = fma(av[j], cospi(2.0 * (double)((j * m) % Q) / Q), acc);
            lam[m] = acc;
        }
        __syncthreads();
        for (int j = tid; j < Q; j += INV_THREADS) {
            double acc = 0.0;
            for (int m = 0; m < Q; m++) acc += cospi(2.0 * (double)((j * m) % Q) / Q) / lam[m];
            bv[j] = acc / Q;
        }
        __syncthreads();
        double *inv = A.ops + (size_t)l * A.stride + off_inv(Q);  // row-major, inv[s][t] = b[(t - s) mod Q]
        for (int e = tid; e < Q * Q; e += INV_THREADS) {
            const int r = e / Q, c = e % Q;
            inv[e] = bv[(c - r + Q) % Q];
        }
        return;
    }
    for (int e = tid; e < Q * Q2; e += INV_THREADS) {
        const int r = e / Q2, c = e % Q2;
        a[r * ld + c] = c < Q ? gent(A, sx, sy, 0.0, 0.0, lx, ly, r, c) : (c - Q == r ? 1.0 : 0.0);
    }
    __syncthreads();
    for (int k = 0; k < Q; k++) {
        if (tid < 32) {  // pivot: largest |a[i][k]| over rows i >= k (lowest row on ties)
            double best = -1.0;
            int bi = k;
            for (int i = k + tid; i < Q; i += 32) {
                const double v = fabs(a[i * ld + k]);
                if (v > best) { best = v; bi = i; }
            }
            for (int o = 16; o; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (tid == 0) s_piv = bi;
        }
        __syncthreads();
        // rows k and p swap, row k is divided by the pivot, and the pivot row
        // is subtracted from every other row to clear column k
        const int p = s_piv;
        const double rp = 1.0 / a[p * ld + k];
        // thread = column tid % 128 (2Q <= 128) and every second row from tid / 128
        const int c = tid & 127;
        if (c < Q2) {
            const double pc = a[p * ld + c] * rp;  // normalised pivot row
            for (int r = tid >> 7; r < Q; r += INV_THREADS / 128) {
                double v;
                if (r == k) {
                    v = pc;
                } else {
                    const int src = r == p ? k : r;
                    v = a[src * ld + c] - a[src * ld + k] * pc;
                }
                nb[r * ld + c] = v;
            }
        }
        __syncthreads();
        double *t = a;
        a = nb;
        nb = t;
    }
    double *inv = A.ops + (size_t)l * A.stride + off_inv(Q);  // row-major
    for (int e = tid; e < Q * Q; e += INV_THREADS) inv[e] = a[(e / Q) * ld + Q + e % Q];
}

// P_o = M2LS_o . Inv_l (far offsets), M2M and L2L compositions; the inverse
// and the kernel-matrix block are staged in shared memory.
// Slots 0..48: M2L offsets (the 3x3 near block skipped); 49..52: M2M of
// child q = slot - 49; 53..56: L2L of child q = slot - 53.  A child's slot
// needs only its Q x Q block of M2MC, so the M2M and L2L work is spread over
// four blocks each, like the offsets.
constexpr int OPS_COMPOSE_SLOTS = 57;
__global__ void k_ops_compose(OpsArgs A) {
    extern __shared__ double sm_c[];
    const int Q = A.Q, l = blockIdx.x, slot = blockIdx.y;
    if (l < 1 || l >= A.L) return;
    if (slot < 49) {
        int ox = slot / 7 - 3, oy = slot % 7 - 3;
        if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1) return;
    }
    if (slot >= 49 && l + 1 >= A.L) return;
    const bool m2m = slot >= 49 && slot < 53, l2l = slot >= 53;
    const int q = m2m ? slot - 49 : slot - 53;  // child (M2M, L2L)
    double *b = A.ops + (size_t)l * A.stride;
    const double *inv = m2m ? A.ops + (size_t)(l + 1) * A.stride + off_inv(Q) : b + off_inv(Q);
    double *iv = sm_c;          // [Q][Q]
    double *mm = sm_c + Q * Q;  // M2LS block, or the child's block of M2MC, [Q][Q]
    for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) iv[e] = inv[e];
    // the kernel-matrix block, evaluated here (class_fmm.py:219-250)
    const double *sx = b + off_small(Q), *sy = sx + A.Qc, *lx = b + off_large(Q), *ly = lx + A.Qc;
    if (slot < 49) {  // M2LS_o[r][t] = G(small_t + o w -> small_r)
        const int ox = slot / 7 - 3, oy = slot % 7 - 3;
        const double w = lvl_width(A, l);
        for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) {
            const int r = e / Q, t = e % Q;
            mm[e] = gent(A, sx, sy, ox * w, oy * w, sx, sy, r, t);
        }
    } else {  // M2MC_l[r][q Q + t] = G(small_{l+1, t} + child offset q -> large_r), child q's block
        const double *b1 = A.ops + (size_t)(l + 1) * A.stride;
        const double *cx = b1 + off_small(Q), *cy = cx + A.Qc;
        const double hw = 0.5 * lvl_width(A, l + 1);
        const double ox = (q >= 2) ? hw : -hw, oy = (q & 1) ? hw : -hw;
        // L2L applies M2MC's transpose (class_fmm.py:329-330): for complex values
        // its real image is built here, as l2l reads this block transposed
        for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) {
            const int r = e / Q, t = e % Q;
            mm[e] = gent(A, cx, cy, ox, oy, lx, ly, r, t, l2l);
        }
    }
    __syncthreads();
    if (slot < 49) {
        double *p = A.poff + ((size_t)l * 49 + slot) * Q * Q;
        for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) {
            int r = e / Q, c = e % Q;
            double s = 0;
            for (int t = 0; t < Q; t++) s = fma(mm[r * Q + t], iv[t * Q + c], s);
            p[e] = s;
        }
    } else if (m2m) {
        double *o = b + off_m2m(Q);  // [4Q cols][Q rows]; this child's columns q Q .. q Q + Q - 1
        for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) {
            int r = e / Q, cc = e % Q;
            double s = 0;
            for (int t = 0; t < Q; t++) s = fma(mm[r * Q + t], iv[t * Q + cc], s);
            o[(size_t)(q * Q + cc) * Q + r] = s;
        }
    } else if (l2l) {
        double *o = b + off_l2l(Q);  // [Q cols][4Q rows]; this child's rows q Q .. q Q + Q - 1
        for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) {
            int rr = e / Q, c = e % Q;
            double s = 0;
            for (int t = 0; t < Q; t++) s = fma(mm[t * Q + rr], iv[t * Q + c], s);
            o[(size_t)c * 4 * Q + q * Q + rr] = s;
        }
    }
}

// directional M2L blocks: for parent direction d = (dx+1)*3 + (dy+1), target
// child a = 2ii+jj and source child b = 2iii+jjj sit at offset
// 2(dx,dy) - (ii,jj) + (iii,jjj) (class_fmm.py:263-283); near offsets are zero.
// rowmax (or null): per (level, row), the largest |value| over all directions
// and columns (bit pattern of a non-negative double, max by atomicMax), for
// the tensor-core M2L's row scales.
__global__ void k_ops_assemble(OpsArgs A, unsigned long long *rowmax) {
    const int Q = A.Q, Q4 = 4 * Q, l = blockIdx.x, d = blockIdx.y;
    if (l < 1 || l >= A.L || d == 4) return;
    int dx = d / 3 - 1, dy = d % 3 - 1;
    double *o = A.ops + (size_t)l * A.stride + off_m2l(Q) + (size_t)d * Q4 * Q4;
    int cur = -1;
    double mx = 0.0;
    for (int e = threadIdx.x; e < Q4 * Q4; e += blockDim.x) {
        int c = e / Q4, r = e % Q4;       // column-major element (r, c)
        int ta = r / Q, rr = r % Q, sb = c / Q, cc = c % Q;
        int ox = 2 * dx - (ta >> 1) + (sb >> 1), oy = 2 * dy - (ta & 1) + (sb & 1);
        double v = 0.0;
        if (!(ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1)) {
            int slot = (ox + 3) * 7 + (oy + 3);
            v = A.poff[((size_t)l * 49 + slot) * Q * Q + rr * Q + cc];
        }
        o[e] = v;
        if (rowmax) {
            if (r != cur) {
                if (cur >= 0) atomicMax(&rowmax[(size_t)l * Q4 + cur], (unsigned long long)__double_as_longlong(mx));
                cur = r;
                mx = 0.0;
            }
            mx = fmax(mx, fabs(v));
        }
    }
    if (rowmax && cur >= 0) atomicMax(&rowmax[(size_t)l * Q4 + cur], (unsigned long long)__double_as_longlong(mx));
}

// Laplace local expansion as a Taylor series about the box centre.  With
// L_k = r2 e^(i theta_k) the equivalent points, z~ = z / w and rho = r2 / w:
//   -(1/2pi) sum_k q_k log|z - L_k| = a0 + Re sum_{j=1..p} c_j z~^j,
//   a0 = -(log r2 / 2pi) sum_k q_k,  c_j = (rho^-j / (2 pi j)) sum_k q_k e^(-i j theta_k),
// valid for |z~| < rho.  taylor_l [(2p+1) rows][Q cols] (column-major) maps the
// downward check potential to (a0, Re c_1, Im c_1, ...) through q = Inv_l u.
__global__ void k_ops_taylor(OpsArgs A, double *taylor, int p) {
    // one block per (level, row): thread k forms C[row][k], thread c the output
    __shared__ double Crow[256];
    const int Q = A.Q, l = blockIdx.x, row = blockIdx.y, R = 2 * p + 1;
    if (l < 1 || l >= A.L || row >= R) return;
    const double *inv = A.ops + (size_t)l * A.stride + off_inv(Q);
    const double w = lvl_width(A, l), r2 = 0.5 * w * A.rf2, rho = r2 / w;
    const double twopi = 2.0 * 3.141592653589793;
    for (int k = threadIdx.x; k < Q; k += blockDim.x) {
        double v;
        if (row == 0) {
            v = -log(r2) / twopi;
        } else {
            int j = (row + 1) / 2;
            double th = (double)((j * k) % Q) * (twopi / Q);  // j theta_k reduced mod 2 pi
            double f = pow(rho, -(double)j) / (twopi * j);
            v = (row & 1) ? f * cos(th) : -f * sin(th);
        }
        Crow[k] = v;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < Q; c += blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < Q; k++) acc = fma(Crow[k], inv[k * Q + c], acc);
        taylor[((size_t)l * Q + c) * R + row] = acc;
    }
}

__global__ void k_to_float(const double *__restrict__ a, float *__restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

void build_operators(kifmm_plan *P) {
    KIFMM_REQUIRE(P->L >= 1 && P->W >= 0, KIFMM_ERR_STATE, "precompute: build_tree first");
    const int L = P->L, Q = P->Q;
    cudaStream_t s = P->stream;
    OpsArgs A{};
    A.L = L; A.Q = Q; A.kind = P->kern.kind; A.k = P->kern.k; A.W = P->W;
    A.circulant = P->opt.e2c == KIFMM_E2C_CIRCULANT;
    A.Qc = P->Qc;
    A.cplx = P->cplx;
    if (P->opt.radii == 1) { A.rf1 = 1.5; A.rf2 = 2.5; }
    else { A.rf1 = std::sqrt(2.0) + 0.01; A.rf2 = 4.0 - std::sqrt(2.0) - 2 * 0.01; }
    A.stride = ops_stride(Q);
    P->ops_stride = A.stride;
    P->ops.alloc(A.stride * (size_t)L);
    KIFMM_CUDA(cudaMemsetAsync(P->ops.p, 0, A.stride * (size_t)L * sizeof(double), s));
    A.ops = P->ops.p;
    DBuf<double> &tmp = P->ops_tmp;
    size_t n49 = (size_t)L * 49 * Q * Q;
    tmp.alloc(n49);
    A.poff = tmp.p;
    for (int l = 0; l < L; l++) {
        double *b = P->ops.p + (size_t)l * A.stride;
        P->lops[l].inv = b + off_inv(Q);
        P->lops[l].m2m = b + off_m2m(Q);
        P->lops[l].l2lT = b + off_l2l(Q);
        P->lops[l].m2lT = b + off_m2l(Q);
        P->lops[l].large = b + off_large(Q);
        P->lops[l].small = b + off_small(Q);
    }
    const bool mixed = P->opt.precision == KIFMM_PREC_MIXED;
    const bool tc = mixed && uses_tensor_m2l(P) && L >= 3;
    unsigned long long *rowmax = nullptr;
    if (tc) {
        P->tc_rowmax.alloc((size_t)L * 4 * Q);
        rowmax = P->tc_rowmax.p;
        KIFMM_CUDA(cudaMemsetAsync(rowmax, 0, (size_t)L * 4 * Q * sizeof(unsigned long long), s));
    }
    // circles + inverse, then kernel matrices composed with the inverses, then
    // the directional M2L blocks (with the row maxima the tensor-core slices use)
    // k_ops_inverse's elimination maps the augmented [E2C | I] row (2Q columns)
    // onto 128 columns per row phase
    KIFMM_REQUIRE(2 * Q <= 128, KIFMM_ERR_ARG, "operator inverse: Nequiv above 64");
    size_t smem = (size_t)2 * Q * (2 * Q + 1) * sizeof(double);
    ensure_dyn_smem(k_ops_inverse, smem);
    k_ops_inverse<<<L, INV_THREADS, smem, s>>>(A);
    KIFMM_LAUNCHED();
    if (P->side && s == P->side) KIFMM_CUDA(cudaEventRecord(P->ops_circ, s));  // circles written
    if (L >= 2) {
        size_t csm = (size_t)5 * Q * Q * sizeof(double);
        ensure_dyn_smem(k_ops_compose, csm);
        k_ops_compose<<<dim3(L, OPS_COMPOSE_SLOTS), 256, csm, s>>>(A);
        KIFMM_LAUNCHED();
        k_ops_assemble<<<dim3(L, 9), 256, 0, s>>>(A, rowmax);
        KIFMM_LAUNCHED();
    }
    if (mixed) {
        if (P->opt.m2l == KIFMM_M2L_FP32) {  // only the FP32 SIMT M2L reads FP32 operators
            P->ops_f.alloc(A.stride * (size_t)L);
            k_to_float<<<grid_for(A.stride * L, 256, 4096), 256, 0, s>>>(P->ops.p, P->ops_f.p, A.stride * (size_t)L);
            KIFMM_LAUNCHED();
        }
        if (tc) build_tc_operators(P);
        if (P->kern.kind == KIFMM_KERNEL_LAPLACE && L >= 3) {
            const int R = 2 * KIFMM_TAYLOR_P + 1;
            P->l2p_taylor.alloc((size_t)L * Q * R);
            KIFMM_REQUIRE(Q <= 256, KIFMM_ERR_ARG, "Nequiv above 256");
            k_ops_taylor<<<dim3(L, R), ((Q + 31) / 32) * 32, 0, s>>>(A, P->l2p_taylor.p, KIFMM_TAYLOR_P);
            KIFMM_LAUNCHED();
        }
    }
    P->have_ops = true;
}

// The operators depend on the kernel, Nequiv, the radii, the root width and the
// number of levels only, so build_tree starts them as soon as the depth is
// known, on the plan's side stream; the rest of the tree build (restriction,
// X-list, entry sort, node tables, with their host round trips) runs meanwhile.
// Buffers allocated here belong to the side stream, which is ordered after all
// earlier work of the main stream, the earlier users of those buffers.  The
// side stream is one per device, shared by all plans (kept until exit), so that
// operator memory freed by one plan is reused by the next in stream order.
void ensure_side(kifmm_plan *P) {
    if (P->side) return;
    P->side = device_side_stream(P->device);
    KIFMM_CUDA(cudaEventCreateWithFlags(&P->ops_fork, cudaEventDisableTiming));
    KIFMM_CUDA(cudaEventCreateWithFlags(&P->ops_done, cudaEventDisableTiming));
    KIFMM_CUDA(cudaEventCreateWithFlags(&P->tree_ev, cudaEventDisableTiming));
    KIFMM_CUDA(cudaEventCreateWithFlags(&P->ops_circ, cudaEventDisableTiming));
}

// fork_recorded: the caller has recorded ops_fork on the main stream at the
// point after which the operators may start (build_tree records it before the
// split-cell kernels, which the operators do not depend on)
void start_operators(kifmm_plan *P, bool fork_recorded) {
    ensure_side(P);
    if (!fork_recorded) KIFMM_CUDA(cudaEventRecord(P->ops_fork, P->stream));
    KIFMM_CUDA(cudaStreamWaitEvent(P->side, P->ops_fork, 0));
    struct Swap {  // launches and allocations go to the side stream meanwhile
        kifmm_plan *P;
        cudaStream_t main, g;
        Swap(kifmm_plan *p) : P(p), main(p->stream), g(g_stream) {
            P->stream = P->side;
            g_stream = P->side;
        }
        ~Swap() {
            P->stream = main;
            g_stream = g;
        }
    } sw(P);
    {
        PhaseScope ph(P, KIFMM_PHASE_OPERATORS);  // events on the side stream
        build_operators(P);
    }
    P->have_ops = false;  // usable once joined
    KIFMM_CUDA(cudaEventRecord(P->ops_done, P->side));
    P->ops_pending = true;
}

// precompute(): the operators count as built; the main stream's wait for the
// side stream is deferred to the first kernel that reads them (the apply
// issues it after its P2M, which needs no operator, so that the operator
// build's tail overlaps the P2M)
void join_operators(kifmm_plan *P) {
    if (!P->ops_pending) return;
    P->ops_pending = false;
    P->ops_wait = P->circ_wait = true;
    P->have_ops = true;
}

void ops_wait_now(kifmm_plan *P) {
    if (!P->ops_wait) return;
    KIFMM_CUDA(cudaStreamWaitEvent(P->stream, P->ops_done, 0));
    P->ops_wait = P->circ_wait = false;
}

// the check circles (written by the first operator kernel) are all the P2M
// reads of the operators
void ops_wait_circles(kifmm_plan *P) {
    if (!P->circ_wait) return;
    KIFMM_CUDA(cudaStreamWaitEvent(P->stream, P->ops_circ, 0));
    P->circ_wait = false;
}

}  // namespace kifmm
