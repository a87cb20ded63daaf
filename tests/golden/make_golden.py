"""Generate the golden fixtures in this folder by running the reference itself.

The reference (dbstein/pykifmm2d, pure Python + numba) ships no tests, golden
vectors or fixtures, so its outputs are pinned here by running its own hot path
(``pykifmm2d/class_fmm.py:166-402`` with ``pykifmm2d/tree.py``) on seeded
inputs and storing what it returns:

* the canonical tree: every node as (level, ix, iy, leaf, fake_leaf, Xlist, ns),
  where ix = (xmin - root_xmin) / width exactly, plus the leaf cell that
  ``Tree.locate_points`` (tree.py:703-727) assigns to every point;
* the potential ``FMM.evaluate_to_points(x, y, True)`` at the sources
  (class_fmm.py:379-399) and, for some cases, at separate targets with
  ``check_self=False``;
* the root box (tree.py:475-484, including its ``ymax = y.min()`` quirk).

The reference does not import on numba 0.65 as shipped: its explicit numba
signatures use the fixed-size array type ``i8[4]`` (tree.py:14,38,71,86). This
script copies the package into a temporary folder and replaces ``i8[4]`` by
``i8[:]`` there; no arithmetic is changed. A fresh ``FMM`` object is used for
every density because a second ``build_expansions`` on one object accumulates
into stale check potentials (tree.py:414 with class_fmm.py:71).

Run from the repository root:
    python tests/golden/make_golden.py [path/to/pykifmm2d]
The reference package folder comes from the argument, else from the
environment variable KIFMM_REFERENCE_PKG; it is only read.  Needs numba.
"""
import os
import shutil
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_package():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KIFMM_REFERENCE_PKG")
    if not ref or not os.path.isfile(os.path.join(ref, "class_fmm.py")):
        sys.exit("usage: make_golden.py <reference pykifmm2d package folder> "
                 "(or set KIFMM_REFERENCE_PKG)")
    return ref


def shimmed_reference():
    tmp = tempfile.mkdtemp(prefix="kifmm_ref_")
    dst = os.path.join(tmp, "pykifmm2d")
    shutil.copytree(reference_package(), dst, ignore=shutil.ignore_patterns("*.pyc", "__pycache__"))
    tp = os.path.join(dst, "tree.py")
    src = open(tp).read()
    assert src.count("i8[4]") >= 4
    open(tp, "w").write(src.replace("i8[4]", "i8[:]"))
    sys.path.insert(0, tmp)
    import pykifmm2d.class_fmm as C  # noqa: E402
    from pykifmm2d.misc.numba_special_functions import _numba_k0  # noqa: E402
    return C, _numba_k0


# --- seeded generators (same RNG call order as the bench generators) -------
def gen_uniform(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.standard_normal(n)


def gen_mixture(n, seed):
    rng = np.random.default_rng(seed)
    nc = int(0.2 * n)
    ng = n - nc
    th = rng.uniform(0, 2 * np.pi, nc)
    cx = rng.uniform(-1, 1, 16)
    cy = rng.uniform(-1, 1, 16)
    sig = 10 ** rng.uniform(-3, -1, 16)
    lab = rng.integers(0, 16, ng)
    x = np.concatenate([cx[lab] + sig[lab] * rng.standard_normal(ng), np.cos(th)])
    y = np.concatenate([cy[lab] + sig[lab] * rng.standard_normal(ng), np.sin(th)])
    return x, y, rng.standard_normal(n)


def gen_annulus(n, seed):
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(0.25, 1, n))
    th = rng.uniform(0, 2 * np.pi, n)
    return r * np.cos(th), r * np.sin(th), rng.uniform(-1, 1, n)


def gen_cluster_dup(n, seed):
    """Uniform background + one tight cluster + a few exact duplicate points."""
    rng = np.random.default_rng(seed)
    nb = int(0.8 * n)
    nc = n - nb - 5
    x = np.concatenate([rng.uniform(-1, 1, nb), 0.3 + 1e-3 * rng.standard_normal(nc)])
    y = np.concatenate([rng.uniform(-1, 1, nb), -0.2 + 1e-3 * rng.standard_normal(nc)])
    pick = rng.choice(x.size, 5, replace=False)
    x = np.concatenate([x, x[pick]])
    y = np.concatenate([y, y[pick]])
    return x, y, rng.standard_normal(n)


def gen_uniform_ctau(n, seed):
    """Uniform points with complex charges N(0,1) + i N(0,1)."""
    rng = np.random.default_rng(seed)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    return x, y, rng.standard_normal(n) + 1j * rng.standard_normal(n)


def gen_circle(n, seed):
    """Points on the unit circle with real charges U(0,1), the set-up of the
    reference's Helmholtz example (examples/hankel.py, test = 'circle')."""
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, 2 * np.pi, n)
    return np.cos(th), np.sin(th), rng.uniform(0, 1, n)


CASES = [
    # name, kernel, k, generator, N, seed, Nequiv, Ncutoff, n_targets
    ("c1_uniform20k", "laplace", 0.0, gen_uniform, 20000, 0, 24, 64, 1000),
    ("mix5k_seed1", "laplace", 0.0, gen_mixture, 5000, 1, 24, 64, 0),
    ("mix20k_seed0", "laplace", 0.0, gen_mixture, 20000, 0, 32, 64, 0),
    ("uniform3k_cut16", "laplace", 0.0, gen_uniform, 3000, 2, 32, 16, 500),
    ("annulus6k_k0", "k0", 10.0, gen_annulus, 6000, 3, 24, 48, 300),
    ("cluster_dup", "laplace", 0.0, gen_cluster_dup, 2500, 5, 20, 20, 0),
    ("mix2k_cut8", "laplace", 0.0, gen_mixture, 2000, 4, 16, 8, 0),
    # complex kernel G = (i/4) H0(k r) with FMM(..., iscomplex=True) (class_fmm.py:174)
    ("helm_uniform6k_k2", "helmholtz", 2.0, gen_uniform_ctau, 6000, 6, 24, 50, 300),
    ("helm_circle4k_k10", "helmholtz", 10.0, gen_circle, 4000, 7, 32, 40, 300),
]


def reference_lists(tree, rank, offs):
    """The reference's interaction lists, read from its own Level arrays and
    walked the way its passes walk them, as canonical row indices
    (rank[offs[l] + i] is the canonical row of node i of level l):

    * colleagues[r, (dx+1)*3 + (dy+1)]: the node of Level.colleagues
      (tree.py:349-375) at cell offset (dx, dy), -1 if none;
    * m2l[k] = (target, source): every block numba_add_interactions adds in
      downward pass 1 (class_fmm.py:323-343): for a node i with
      doit = (not_leaf | Xlist) & ~fake_leaf and a colleague ci != i whose child
      group has a density (parent_density_ind[trunc(children_ind[ci] / 4)] >= 0),
      child k of i receives child b of that group unless the CM2LS block for
      (k, b) is zeroed as near (class_fmm.py:266-291);
    * p2p[k] = (leaf, source): numba_target_neighbor_evaluation
      (class_fmm.py:90-111) at the sources: each leaf that holds a point reads
      every colleague with ns > 0.
    """
    root = float(tree.xmin)
    coll_rows, m2l, p2p = [], [], []
    for l, L in enumerate(tree.Levels):
        w = L.width
        ix = np.rint((L.xmin - root) / w).astype(np.int64)
        iy = np.rint((L.ymin - root) / w).astype(np.int64)
        C = -np.ones((L.n_node, 9), dtype=np.int64)
        for i in range(L.n_node):
            for c in L.colleagues[i]:
                if c >= 0:
                    C[i, (ix[c] - ix[i] + 1) * 3 + (iy[c] - iy[i] + 1)] = rank[offs[l] + c]
        coll_rows.append(C)
        ns = L.top_ind - L.bot_ind
        for i in np.nonzero(L.leaf & (ns > 0))[0]:
            for c in L.colleagues[i]:
                if c >= 0 and ns[c] > 0:
                    p2p.append((rank[offs[l] + i], rank[offs[l] + c]))
        if l < 1 or l > tree.levels - 2:
            continue
        D = tree.Levels[l + 1]
        doit = (~L.leaf | L.Xlist) & ~L.fake_leaf
        ci4 = (L.children_ind / 4).astype(int)
        for i in np.nonzero(doit)[0]:
            for ci in L.colleagues[i]:
                if ci < 0 or ci == i:
                    continue
                xd = int(np.sign(L.xmid[ci] - L.xmid[i]))
                yd = int(np.sign(L.ymid[ci] - L.ymid[i]))
                if D.parent_density_ind[ci4[ci]] < 0:
                    continue
                for k in range(4):
                    for b in range(4):
                        ox = 2 * xd - (k >> 1) + (b >> 1)
                        oy = 2 * yd - (k & 1) + (b & 1)
                        if abs(ox) <= 1 and abs(oy) <= 1:
                            continue
                        m2l.append((rank[offs[l + 1] + 4 * ci4[i] + k], rank[offs[l + 1] + 4 * ci4[ci] + b]))
    coll = np.concatenate(coll_rows, axis=0)
    out_coll = np.empty_like(coll)
    out_coll[rank] = coll
    m2l = np.array(sorted(m2l), dtype=np.int64).reshape(-1, 2)
    p2p = np.array(sorted(p2p), dtype=np.int64).reshape(-1, 2)
    return out_coll, m2l, p2p


def canonical_tree(tree, x, y):
    root = float(tree.xmin)
    rows = []
    for l, L in enumerate(tree.Levels):
        w = L.width
        ix = np.rint((L.xmin - root) / w).astype(np.int64)
        iy = np.rint((L.ymin - root) / w).astype(np.int64)
        assert np.all(root + ix * w == L.xmin) and np.all(root + iy * w == L.ymin)
        xl = L.Xlist.astype(np.int64)
        ns = (L.top_ind - L.bot_ind).astype(np.int64)
        rows.append(np.stack([np.full(L.n_node, l), ix, iy, L.leaf.astype(np.int64),
                              L.fake_leaf.astype(np.int64), xl, ns], axis=1))
        # colleague lists are exactly "all same-level nodes within one cell"
        cells = {(a, b): i for i, (a, b) in enumerate(zip(ix, iy))}
        for i in range(L.n_node):
            got = set(int(c) for c in L.colleagues[i] if c >= 0)
            want = set(j for dx in (-1, 0, 1) for dy in (-1, 0, 1)
                       for j in [cells.get((ix[i] + dx, iy[i] + dy))] if j is not None)
            assert got == want, (l, i, got, want)
    nodes = np.concatenate(rows, axis=0)
    inds, locs = tree.locate_points(x, y)
    pl = np.zeros((x.size, 3), dtype=np.int64)
    for l, L in enumerate(tree.Levels):
        m = inds == l
        w = L.width
        pl[m, 0] = l
        pl[m, 1] = np.rint((L.xmin[locs[m]] - root) / w).astype(np.int64)
        pl[m, 2] = np.rint((L.ymin[locs[m]] - root) / w).astype(np.int64)
    order = np.lexsort((nodes[:, 2], nodes[:, 1], nodes[:, 0]))
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    offs = np.concatenate([[0], np.cumsum([L.n_node for L in tree.Levels])])
    lists = reference_lists(tree, rank, offs)
    return nodes[order], pl, lists


def main():
    import numba
    C, k0 = shimmed_reference()

    @numba.njit("f8(f8,f8,f8,f8)", fastmath=True)
    def laplace_eval(sx, sy, tx, ty):
        return -0.25 / np.pi * np.log((tx - sx) ** 2 + (ty - sy) ** 2)

    # H0 from the C library's Bessel functions J0, Y0 (the reference's example
    # interpolates scipy's hankel1 with fast_interp, which is not installed)
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    j0, y0 = libm.j0, libm.y0
    for f in (j0, y0):
        f.restype = ctypes.c_double
        f.argtypes = [ctypes.c_double]

    def helmholtz_factory(kk):
        @numba.njit("c16(f8,f8,f8,f8)", fastmath=True)
        def h_eval(sx, sy, tx, ty):
            z = kk * np.sqrt((tx - sx) ** 2 + (ty - sy) ** 2)
            return 0.25j * (j0(z) + 1j * y0(z))
        return h_eval

    def k0_factory(kk):
        @numba.njit("f8(f8,f8,f8,f8)", fastmath=True)
        def k0_eval(sx, sy, tx, ty):
            return k0(kk * np.sqrt((tx - sx) ** 2 + (ty - sy) ** 2)) / (2 * np.pi)
        return k0_eval

    for name, kern, kk, gen, n, seed, neq, cut, ntarg in CASES:
        cplx = kern == "helmholtz"
        ke = {"laplace": laplace_eval, "k0": None, "helmholtz": None}[kern]
        if kern == "k0":
            ke = k0_factory(kk)
        elif cplx:
            ke = helmholtz_factory(kk)
        nf = C.prepare_numba_functions_on_the_fly(ke)
        kf = C.Get_Kernel_Functions(ke)
        x, y, tau = gen(n, seed)
        t0 = time.time()
        f = C.FMM(x, y, kf, nf, neq, cut, cplx)
        f.build_tree()
        f.precompute()
        f.build_expansions(tau)
        pot = f.evaluate_to_points(x, y, True)
        dt = time.time() - t0
        nodes, pl, (coll, m2l, p2p) = canonical_tree(f.tree, x, y)
        out = dict(x=x, y=y, tau=tau, pot=pot, nodes=nodes, point_leaf=pl,
                   colleagues=coll, m2l_pairs=m2l, p2p_pairs=p2p,
                   kernel=np.array({"laplace": 0, "k0": 1, "helmholtz": 2}[kern]), k=np.array(kk),
                   nequiv=np.array(neq), ncutoff=np.array(cut),
                   root=np.array([f.tree.xmin, f.tree.xmax], dtype=np.float64),
                   levels=np.array(f.tree.levels))
        if ntarg:
            rng = np.random.default_rng(1000 + seed)
            lo, hi = float(f.tree.xmin), float(f.tree.xmax)
            xt = rng.uniform(max(lo, x.min()), min(hi, x.max()), ntarg)
            yt = rng.uniform(max(lo, y.min()), min(hi, y.max()), ntarg)
            out.update(xt=xt, yt=yt, pot_targets=f.evaluate_to_points(xt, yt, False))
        # FP64 direct sum (the reference's KAS, class_fmm.py:134-143) for information
        KF, KA, KAS = kf
        ref = np.zeros(n, dtype=complex if cplx else float)
        KAS(x, y, tau, ref)
        fin = np.isfinite(ref)  # coincident points make the i != j direct sum infinite
        err = np.abs(pot - ref)[fin].max() / np.abs(ref[fin]).max()
        out["direct"] = ref
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(f"{name}: N={n} levels={f.tree.levels} nodes={nodes.shape[0]} "
              f"m2l_pairs={m2l.shape[0]} p2p_pairs={p2p.shape[0]} "
              f"leaves={int(nodes[:,3].sum())} fake={int(nodes[:,4].sum())} "
              f"xlist={int(nodes[:,5].sum())} ref_time={dt:.2f}s relerr_vs_direct={err:.2e}",
              flush=True)


if __name__ == "__main__":
    main()
