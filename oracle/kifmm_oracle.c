/*
 * kifmm_oracle.c -- CPU restatement of the reference's adaptive 2D KIFMM.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the checker that the
 * tests, the smoke check and the CPU-baseline leg of bench.py compare the
 * CUDA path against.  Nothing in the product links or calls it.
 *
 * It restates, step for step, the algorithm of dbstein/pykifmm2d's live FMM
 * (pykifmm2d/class_fmm.py:166-402 over pykifmm2d/tree.py:460-590):
 *   - tree build by level splitting with the same in-place 4-way partition,
 *     the same colleague tagging, level restriction and X-list fake leaves;
 *   - operator precompute (E2C LU, M2MC, M2LS, CM2LS) per level;
 *   - upward pass (M2M + P2M + LU solve), downward pass (L2L + M2L GEMMs +
 *     scatter), local expansions, L2P and P2P evaluation.
 * Loops the reference runs under numba.prange run under OpenMP here.
 *
 * The modified-Helmholtz K0 used here is computed independently of any
 * table: the power series of K0 for x < 2 and the trapezoidal rule on the
 * integral K0(x) = int_0^inf exp(-x cosh t) dt (DLMF 10.32.9) for x >= 2.
 * The complex mode (the reference's FMM(..., iscomplex=True)) runs the same
 * FMM on complex values (kifmm_oracle_fmm.inc, entry points orkc_*), with
 * the Helmholtz kernel (i/4) H0(k r) = (i/4) (J0(k r) + i Y0(k r)) from the C
 * library's Bessel functions.
 */
#define _DEFAULT_SOURCE  /* j0, y0 (POSIX Bessel functions) */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define ORK_MAXLEV 64
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ kernels */
static double ork_k0(double x)
{
    if (x < 0) return NAN;
    if (x == 0) return INFINITY;
    if (x < 2.0) {
        /* K0(x) = -(ln(x/2)+gamma) I0(x) + sum_{k>=1} H_k (x^2/4)^k/(k!)^2 */
        const double g = 0.57721566490153286060651209;
        double q = 0.25 * x * x, term = 1.0, i0 = 1.0, s = 0.0, hk = 0.0;
        for (int k = 1; k < 40; k++) {
            term *= q / ((double)k * (double)k);
            hk += 1.0 / k;
            i0 += term;
            s += hk * term;
            if (term < 1e-18) break;
        }
        return -(log(0.5 * x) + g) * i0 + s;
    }
    /* trapezoidal rule, exponentially convergent for this analytic integrand */
    /* step small enough for the Gaussian-like peak of width ~ 1/sqrt(x) */
    const double h = fmin(0.125, 0.5 / sqrt(x));
    double acc = 0.5; /* f(0) / 2 with f(t) = exp(-x (cosh t - 1)) */
    for (int j = 1; j < 4000; j++) {
        double f = exp(-x * (cosh(j * h) - 1.0));
        acc += f;
        if (f < 1e-19) break;
    }
    return exp(-x) * h * acc;
}

typedef struct { int kind; double k; } OKern;

static int isgn(double v) { return (v > 0) - (v < 0); }

/* G(s -> t): Laplace -log(r^2)/(4 pi); modified Helmholtz K0(k r)/(2 pi).
 * The reference plug-ins: examples/laplace2.py:31-36, modified_helmholtz.py:38-43. */
static inline double ork_eval(OKern kn, double sx, double sy, double tx, double ty)
{
    double dx = tx - sx, dy = ty - sy;
    double r2 = dx * dx + dy * dy;
    if (kn.kind == 0) return -0.25 / M_PI * log(r2);
    return ork_k0(kn.k * sqrt(r2)) / (2.0 * M_PI);
}

/* ------------------------------------------------------------------- levels */
typedef struct {
    int64_t n;
    double width, half;
    double *xmin, *ymin, *xmid, *ymid;
    int64_t *bot, *top, *parent, *children;
    uint8_t *leaf, *fake, *xlist, *cu;
    int64_t *coll;           /* n x 9, -1 padded */
    int64_t *depth, ndepth;  /* ndepth lags n after X-list fake nodes */
    int64_t n_alloc, n_sib;
    int64_t *pdi, *tdi;      /* parent_density_ind [n/4], this_density_ind [n] */
} OLevel;

typedef struct {
    int64_t N, ppl;
    double *x, *y;
    int64_t *ordv;
    double rmin, rmax;
    int L;
    OLevel lv[ORK_MAXLEV];
} OTree;

static void *xrealloc(void *p, size_t sz) { void *q = realloc(p, sz ? sz : 1); if (!q) abort(); return q; }

static void level_basic(OLevel *v)
{
    v->xmid = xrealloc(v->xmid, v->n * sizeof(double));
    v->ymid = xrealloc(v->ymid, v->n * sizeof(double));
    for (int64_t i = 0; i < v->n; i++) {
        v->xmid[i] = v->xmin[i] + v->half;
        v->ymid[i] = v->ymin[i] + v->half;
    }
}

/* Level.__init__ (tree.py:318-338) and Level.add_nodes (tree.py:384-395) */
static void level_append(OLevel *v, int64_t m, const double *xmin, const double *ymin,
                         const int64_t *bot, const int64_t *top, const int64_t *par, int xl)
{
    int64_t n0 = v->n, n = n0 + m;
    v->xmin = xrealloc(v->xmin, n * sizeof(double));
    v->ymin = xrealloc(v->ymin, n * sizeof(double));
    v->bot = xrealloc(v->bot, n * sizeof(int64_t));
    v->top = xrealloc(v->top, n * sizeof(int64_t));
    v->parent = xrealloc(v->parent, n * sizeof(int64_t));
    v->children = xrealloc(v->children, n * sizeof(int64_t));
    v->leaf = xrealloc(v->leaf, n);
    v->fake = xrealloc(v->fake, n);
    for (int64_t i = 0; i < m; i++) {
        v->xmin[n0 + i] = xmin[i];
        v->ymin[n0 + i] = ymin[i];
        v->bot[n0 + i] = bot[i];
        v->top[n0 + i] = top[i];
        v->parent[n0 + i] = par[i];
        v->children[n0 + i] = -1;
        v->leaf[n0 + i] = xl ? 0 : 1;
        v->fake[n0 + i] = xl ? 1 : 0;
    }
    v->n = n;
    level_basic(v);
}

/* classify + get_inds + get_target + reorder_inplace (tree.py:14-126):
 * class = 2*(x > midx) + (y > midy); in-place cycle placement. */
static void reorder_inplace(double *x, double *y, int64_t *ordv, int64_t n,
                            double midx, double midy, int64_t nns[4])
{
    int8_t *cl = malloc(n ? n : 1);
    int64_t ns[4] = {0, 0, 0, 0}, inds[4];
    for (int64_t i = 0; i < n; i++) {
        int c = 2 * (x[i] > midx) + (y[i] > midy);
        cl[i] = (int8_t)c;
        ns[c]++;
    }
    inds[0] = 0;
    for (int i = 0; i < 3; i++) inds[i + 1] = inds[i] + ns[i];
    for (int i = 0; i < 4; i++) nns[i] = inds[i];
    for (int64_t i = 0; i < n; i++) {
        int target = i < nns[1] ? 0 : i < nns[2] ? 1 : i < nns[3] ? 2 : 3;
        for (;;) {
            int cli = cl[i];
            int64_t icli = inds[cli];
            if (cli != target) {
                int8_t tc = cl[i]; cl[i] = cl[icli]; cl[icli] = tc;
                double td = x[i]; x[i] = x[icli]; x[icli] = td;
                td = y[i]; y[i] = y[icli]; y[icli] = td;
                int64_t to = ordv[i]; ordv[i] = ordv[icli]; ordv[icli] = to;
                inds[cli]++;
                if (cl[icli] == target) break;
            } else {
                inds[target]++;
                break;
            }
        }
    }
    free(cl);
}

/* divide_and_reorder (tree.py:128-190) followed by appending the children to
 * the next level (get_new_level tree.py:229-258 / split_bad_leaves :296-311). */
static void divide_into(OTree *t, int l, const uint8_t *tosplit, int xl)
{
    OLevel *v = &t->lv[l], *d = &t->lv[l + 1];
    int64_t nsplit = 0;
    int64_t *ids = malloc((v->n ? v->n : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < v->n; i++) { ids[i] = nsplit; if (tosplit[i]) nsplit++; }
    int64_t m = 4 * nsplit;
    double *xmin = malloc((m ? m : 1) * sizeof(double)), *ymin = malloc((m ? m : 1) * sizeof(double));
    int64_t *bot = malloc((m ? m : 1) * sizeof(int64_t)), *top = malloc((m ? m : 1) * sizeof(int64_t));
    int64_t *par = malloc((m ? m : 1) * sizeof(int64_t));
    int64_t start = d->n;
    double hw = v->half;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < v->n; i++) {
        if (!tosplit[i]) continue;
        int64_t s = ids[i], bi = v->bot[i], ti = v->top[i], nns[4];
        reorder_inplace(t->x + bi, t->y + bi, t->ordv + bi, ti - bi, v->xmid[i], v->ymid[i], nns);
        xmin[4 * s + 0] = v->xmid[i] - hw; xmin[4 * s + 1] = v->xmid[i] - hw;
        xmin[4 * s + 2] = v->xmid[i];      xmin[4 * s + 3] = v->xmid[i];
        ymin[4 * s + 0] = v->ymid[i] - hw; ymin[4 * s + 1] = v->ymid[i];
        ymin[4 * s + 2] = v->ymid[i] - hw; ymin[4 * s + 3] = v->ymid[i];
        for (int j = 0; j < 4; j++) bot[4 * s + j] = bi + nns[j];
        top[4 * s + 0] = bi + nns[1]; top[4 * s + 1] = bi + nns[2];
        top[4 * s + 2] = bi + nns[3]; top[4 * s + 3] = ti;
        if (!xl) v->leaf[i] = 0;
        for (int j = 0; j < 4; j++) par[4 * s + j] = i;
        v->children[i] = start + 4 * s;
    }
    d->width = v->half;
    d->half = 0.5 * d->width;
    level_append(d, m, xmin, ymin, bot, top, par, xl);
    free(ids); free(xmin); free(ymin); free(bot); free(top); free(par);
}

/* Level.tag_colleagues (tree.py:349-375): direct O(n^2) below 100 nodes
 * (numba_tag_colleagues :260-272), otherwise via the parent's colleagues'
 * children (numba_loop_colleagues :274-294). */
static void tag_colleagues(OTree *t, int l)
{
    OLevel *v = &t->lv[l];
    v->coll = xrealloc(v->coll, (v->n ? v->n : 1) * 9 * sizeof(int64_t));
    for (int64_t i = 0; i < 9 * v->n; i++) v->coll[i] = -1;
    double dist = 1.5 * v->width, dist2 = dist * dist;
    if (v->n < 100) {
#pragma omp parallel for
        for (int64_t i = 0; i < v->n; i++) {
            int it = 0;
            for (int64_t j = 0; j < v->n; j++) {
                double dx = v->xmid[i] - v->xmid[j], dy = v->ymid[i] - v->ymid[j];
                if (dx * dx + dy * dy < dist2) v->coll[9 * i + it++] = j;
            }
        }
        return;
    }
    OLevel *a = &t->lv[l - 1];
#pragma omp parallel for
    for (int64_t i = 0; i < v->n; i++) {
        int it = 0;
        int64_t pi = v->parent[i];
        for (int j = 0; j < 9; j++) {
            int64_t pij = a->coll[9 * pi + j];
            if (pij < 0 || a->children[pij] < 0) continue;
            for (int k = 0; k < 4; k++) {
                int64_t c = a->children[pij] + k;
                double dx = v->xmid[i] - v->xmid[c], dy = v->ymid[i] - v->ymid[c];
                if (dx * dx + dy * dy < dist2) v->coll[9 * i + it++] = c;
            }
        }
    }
}

/* gather_depths (tree.py:582-585) with numba_get_depths (:423-430) */
static void gather_depths(OTree *t)
{
    for (int l = t->L - 1; l >= 0; l--) {
        OLevel *v = &t->lv[l];
        v->depth = xrealloc(v->depth, (v->n ? v->n : 1) * sizeof(int64_t));
        v->ndepth = v->n;
        for (int64_t i = 0; i < v->n; i++) v->depth[i] = 0;
        if (l == t->L - 1) continue;
        OLevel *d = &t->lv[l + 1];
        for (int64_t i = 0; i < v->n; i++) {
            if (v->leaf[i]) continue;
            int64_t c = v->children[i], mx = d->depth[c];
            for (int k = 1; k < 4; k++) if (d->depth[c + k] > mx) mx = d->depth[c + k];
            v->depth[i] = mx + 1;
        }
    }
}

void ork_tree_free(OTree *t)
{
    if (!t) return;
    for (int l = 0; l < ORK_MAXLEV; l++) {
        OLevel *v = &t->lv[l];
        free(v->xmin); free(v->ymin); free(v->xmid); free(v->ymid);
        free(v->bot); free(v->top); free(v->parent); free(v->children);
        free(v->leaf); free(v->fake); free(v->xlist); free(v->cu);
        free(v->coll); free(v->depth); free(v->pdi); free(v->tdi);
    }
    free(t->x); free(t->y); free(t->ordv);
    free(t);
}

/* Tree.__init__ (tree.py:464-522).  fix_bbox = 0 keeps the reference's root
 * box [floor(min(xmin, ymin)), ceil(max(xmax, ymin))] (tree.py:475-484). */
int ork_tree_build(const double *x, const double *y, int64_t N, int64_t ppl, int fix_bbox, OTree **out)
{
    if (N <= 0 || ppl <= 0) return 1;
    OTree *t = calloc(1, sizeof(OTree));
    t->N = N; t->ppl = ppl;
    t->x = malloc(N * sizeof(double)); t->y = malloc(N * sizeof(double));
    t->ordv = malloc(N * sizeof(int64_t));
    memcpy(t->x, x, N * sizeof(double)); memcpy(t->y, y, N * sizeof(double));
    double xmn = x[0], xmx = x[0], ymn = y[0], ymx = y[0];
    for (int64_t i = 0; i < N; i++) {
        if (!isfinite(x[i]) || !isfinite(y[i])) { ork_tree_free(t); return 2; }
        if (x[i] < xmn) xmn = x[i];
        if (x[i] > xmx) xmx = x[i];
        if (y[i] < ymn) ymn = y[i];
        if (y[i] > ymx) ymx = y[i];
        t->ordv[i] = i;
    }
    double ytop = fix_bbox ? ymx : ymn;
    t->rmin = floor(xmn < ymn ? xmn : ymn);
    t->rmax = ceil(xmx > ytop ? xmx : ytop);
    OLevel *v0 = &t->lv[0];
    v0->width = t->rmax - t->rmin;
    v0->half = 0.5 * v0->width;
    double r = t->rmin; int64_t b = 0, tp = N, p = -1;
    level_append(v0, 1, &r, &r, &b, &tp, &p, 0);
    t->L = 1;
    if (N > ppl) {
        for (;;) {
            OLevel *v = &t->lv[t->L - 1];
            uint8_t *ts = malloc(v->n);
            int64_t cnt = 0;
            for (int64_t i = 0; i < v->n; i++) { ts[i] = (v->top[i] - v->bot[i]) > ppl; cnt += ts[i]; }
            if (t->L >= ORK_MAXLEV - 1) { free(ts); ork_tree_free(t); return 3; }
            divide_into(t, t->L - 1, ts, 0);
            free(ts);
            t->L++;
            OLevel *d = &t->lv[t->L - 1];
            int more = 0;
            for (int64_t i = 0; i < d->n; i++) if (d->top[i] - d->bot[i] > ppl) { more = 1; break; }
            if (!more) break;
        }
    }
    for (int l = 0; l < t->L; l++) tag_colleagues(t, l);
    gather_depths(t);
    /* level_restrict (tree.py:533-545) with numba_get_bads (:432-444) */
    int64_t newn = 1;
    while (newn > 0) {
        newn = 0;
        for (int l = 1; l < t->L - 2; l++) {
            OLevel *v = &t->lv[l];
            uint8_t *bads = calloc(v->n ? v->n : 1, 1);
            int64_t nb = 0;
            for (int64_t i = 0; i < v->n; i++) {
                if (!v->leaf[i]) continue;
                for (int j = 0; j < 9; j++) {
                    int64_t cj = v->coll[9 * i + j];
                    if (cj < 0) continue;
                    int64_t dd = v->depth[i] - v->depth[cj];
                    if (dd > 1 || dd < -1) { bads[i] = 1; }
                }
                nb += bads[i];
            }
            divide_into(t, l, bads, 0);
            tag_colleagues(t, l + 1);
            gather_depths(t);
            free(bads);
            newn += nb;
        }
    }
    /* split_Xlist (tree.py:546-576) with numba_get_Xlist (:446-458) */
    for (int l = 0; l < t->L; l++) {
        OLevel *v = &t->lv[l];
        v->xlist = xrealloc(v->xlist, v->n ? v->n : 1);
        memset(v->xlist, 0, v->n);
        if (l > 0 && l < t->L - 1) {
            int64_t nd = v->ndepth, nx = 0;
            for (int64_t i = 0; i < nd; i++) {
                if (!v->leaf[i]) continue;
                for (int j = 0; j < 9; j++) {
                    int64_t cj = v->coll[9 * i + j];
                    if (cj >= 0 && cj < nd && v->depth[i] - v->depth[cj] < 0) v->xlist[i] = 1;
                }
                nx += v->xlist[i];
            }
            if (nx > 0) {
                divide_into(t, l, v->xlist, 1);
                tag_colleagues(t, l + 1);
            }
        }
        if (l > 0) {
            v->cu = xrealloc(v->cu, v->n);
            v->pdi = xrealloc(v->pdi, (v->n / 4 ? v->n / 4 : 1) * sizeof(int64_t));
            v->tdi = xrealloc(v->tdi, v->n * sizeof(int64_t));
            for (int64_t i = 0; i < v->n; i++)
                v->cu[i] = ((v->leaf[i] && !v->xlist[i]) || v->fake[i]) && (v->top[i] > v->bot[i]);
            int64_t ns = 0, na = 0;
            for (int64_t g = 0; g < v->n / 4; g++) {
                int has = 0;
                for (int k = 0; k < 4; k++) has |= v->top[4 * g + k] > v->bot[4 * g + k];
                v->pdi[g] = has ? ns++ : -1;
                for (int k = 0; k < 4; k++) v->tdi[4 * g + k] = has ? na++ : -1;
            }
            v->n_sib = ns;
            v->n_alloc = na;
        }
    }
    *out = t;
    return 0;
}

int ork_tree_levels(const OTree *t) { return t->L; }

int64_t ork_tree_num_nodes(const OTree *t)
{
    int64_t s = 0;
    for (int l = 0; l < t->L; l++) s += t->lv[l].n;
    return s;
}

/* Canonical export: per node (level, ix, iy, leaf, fake_leaf, Xlist, ns) with
 * ix = (xmin - root) / width (exact on the dyadic grid). */
void ork_tree_export(const OTree *t, int64_t *nodes, double *root)
{
    int64_t r = 0;
    for (int l = 0; l < t->L; l++) {
        const OLevel *v = &t->lv[l];
        for (int64_t i = 0; i < v->n; i++, r++) {
            nodes[7 * r + 0] = l;
            nodes[7 * r + 1] = (int64_t)llround((v->xmin[i] - t->rmin) / v->width);
            nodes[7 * r + 2] = (int64_t)llround((v->ymin[i] - t->rmin) / v->width);
            nodes[7 * r + 3] = v->leaf[i];
            nodes[7 * r + 4] = v->fake[i];
            nodes[7 * r + 5] = v->xlist ? v->xlist[i] : 0;
            nodes[7 * r + 6] = v->top[i] - v->bot[i];
        }
    }
    root[0] = t->rmin;
    root[1] = t->rmax;
}

/* ------------------------------------------------------- interaction lists
 * Node numbers below are export rows (ork_tree_export order). */
static int64_t level_offset(const OTree *t, int l)
{
    int64_t o = 0;
    for (int k = 0; k < l; k++) o += t->lv[k].n;
    return o;
}

/* Level.colleagues (tree.py:349-375) by direction: coll[r][(dx+1)*3+(dy+1)]
 * is the colleague at cell offset (dx, dy), -1 if none. */
void ork_tree_colleagues(const OTree *t, int64_t *coll)
{
    for (int l = 0; l < t->L; l++) {
        const OLevel *v = &t->lv[l];
        int64_t off = level_offset(t, l);
        for (int64_t i = 0; i < v->n; i++) {
            int64_t *row = coll + 9 * (off + i);
            for (int j = 0; j < 9; j++) row[j] = -1;
            for (int j = 0; j < 9; j++) {
                int64_t c = v->coll[9 * i + j];
                if (c < 0) continue;
                int64_t dx = llround((v->xmin[c] - v->xmin[i]) / v->width);
                int64_t dy = llround((v->ymin[c] - v->ymin[i]) / v->width);
                row[(dx + 1) * 3 + (dy + 1)] = off + c;
            }
        }
    }
}

/* The (target, source) node pairs of downward pass 1's M2L as
 * numba_add_interactions adds them (class_fmm.py:17-33, :323-343): for a node
 * with doit = (!leaf || Xlist) && !fake and a colleague ci != i whose child
 * group has a density (parent_density_ind[trunc(children[ci] / 4)] >= 0),
 * child k of i receives child b of that group unless block (k, b) of the
 * directional CM2LS is zeroed as near.  pairs may be NULL (count only). */
int64_t ork_m2l_pairs(const OTree *t, int64_t *pairs)
{
    int64_t n = 0;
    for (int l = 1; l < t->L - 1; l++) {
        const OLevel *v = &t->lv[l], *d = &t->lv[l + 1];
        int64_t off1 = level_offset(t, l + 1);
        for (int64_t i = 0; i < v->n; i++) {
            int doit = (!v->leaf[i] || v->xlist[i]) && !v->fake[i];
            if (!doit) continue;
            for (int j = 0; j < 9; j++) {
                int64_t ci = v->coll[9 * i + j];
                if (ci < 0 || ci == i) continue;
                int xd = isgn(v->xmid[ci] - v->xmid[i]), yd = isgn(v->ymid[ci] - v->ymid[i]);
                if (d->pdi[v->children[ci] / 4] < 0) continue;
                for (int k = 0; k < 4; k++)
                    for (int b = 0; b < 4; b++) {
                        int ox = 2 * xd - (k >> 1) + (b >> 1), oy = 2 * yd - (k & 1) + (b & 1);
                        if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1) continue;
                        if (pairs) {
                            pairs[2 * n] = off1 + 4 * (v->children[i] / 4) + k;
                            pairs[2 * n + 1] = off1 + 4 * (v->children[ci] / 4) + b;
                        }
                        n++;
                    }
            }
        }
    }
    return n;
}

/* The (leaf, source) node pairs of the near field at the sources
 * (numba_target_neighbor_evaluation, class_fmm.py:90-111): every leaf that
 * holds a point reads each colleague with points.  pairs may be NULL. */
int64_t ork_p2p_pairs(const OTree *t, int64_t *pairs)
{
    int64_t n = 0;
    for (int l = 0; l < t->L; l++) {
        const OLevel *v = &t->lv[l];
        int64_t off = level_offset(t, l);
        for (int64_t i = 0; i < v->n; i++) {
            if (!v->leaf[i] || v->top[i] <= v->bot[i]) continue;
            for (int j = 0; j < 9; j++) {
                int64_t c = v->coll[9 * i + j];
                if (c < 0 || v->top[c] <= v->bot[c]) continue;
                if (pairs) { pairs[2 * n] = off + i; pairs[2 * n + 1] = off + c; }
                n++;
            }
        }
    }
    return n;
}

/* locate_points (tree.py:703-727): descend with strict '>' until a leaf. */
static void locate1(const OTree *t, double x, double y, int *ind, int64_t *loc)
{
    int l = 0;
    int64_t i = 0;
    while (!t->lv[l].leaf[i]) {
        int64_t c = t->lv[l].children[i];
        if (x > t->lv[l].xmid[i]) c += 2;
        if (y > t->lv[l].ymid[i]) c += 1;
        i = c;
        l++;
    }
    *ind = l;
    *loc = i;
}

void ork_locate(const OTree *t, const double *x, const double *y, int64_t n, int64_t *out)
{
#pragma omp parallel for
    for (int64_t p = 0; p < n; p++) {
        int l; int64_t i;
        locate1(t, x[p], y[p], &l, &i);
        const OLevel *v = &t->lv[l];
        out[3 * p + 0] = l;
        out[3 * p + 1] = (int64_t)llround((v->xmin[i] - t->rmin) / v->width);
        out[3 * p + 2] = (int64_t)llround((v->ymin[i] - t->rmin) / v->width);
    }
}

/* ------------------------------------------------- the FMM, real and complex */
/* Helmholtz G(s -> t) = (i/4) H0^(1)(k |t - s|) (examples/hankel.py:37-39);
 * the real kernels promoted to complex values otherwise. */
#define ORK_KERNEL_HELMHOLTZ 2
static inline double complex orkc_eval(OKern kn, double sx, double sy, double tx, double ty)
{
    if (kn.kind == ORK_KERNEL_HELMHOLTZ) {
        double dx = tx - sx, dy = ty - sy, z = kn.k * sqrt(dx * dx + dy * dy);
        return 0.25 * I * (j0(z) + I * y0(z));
    }
    return ork_eval(kn, sx, sy, tx, ty);
}

#define OV double
#define OP(name) ork_##name
#define OABS(v) fabs(v)
#define OEVAL ork_eval
#define OFMM_T ork_fmm_t
#include "kifmm_oracle_fmm.inc"
#undef OV
#undef OP
#undef OABS
#undef OEVAL
#undef OFMM_T

#define OV double complex
#define OP(name) orkc_##name
#define OABS(v) cabs(v)
#define OEVAL orkc_eval
#define OFMM_T orkc_fmm_t
#include "kifmm_oracle_fmm.inc"
#undef OV
#undef OP
#undef OABS
#undef OEVAL
#undef OFMM_T

double ork_k0_value(double x) { return ork_k0(x); }
void ork_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int ork_max_threads(void) { return omp_get_max_threads(); }
