"""GPU parity at the benchmark configurations' own sizes, and the interaction
lists.

* Lists: the CUDA path's colleague lists, M2L (target, source) pairs and P2P
  (leaf, source) pairs (``kifmm_export_lists``) against the lists read from
  the reference's own Level arrays (tests/golden, make_golden.reference_lists)
  and against the oracle.  Colleagues and P2P pairs are equal.  The M2L pairs
  are the reference's minus exactly those whose target is a fake leaf: the
  reference computes M2L into the fake children of X-list leaves
  (class_fmm.py:325 includes Xlist in ``doit``) but never reads them -- no
  point is located in a fake leaf (tree.py:712-727 stops at the X-list leaf)
  and fake leaves pass nothing down (they are excluded from ``doit``).
* Full size: the 1M Gaussian mixture + circle (Nequiv 32), the 4M uniform
  cloud (Nequiv 32) and the 2M K0 annulus (k = 10, Nequiv 40, Ncutoff 48)
  are built on the GPU; the tree (node set, flags, counts, point-to-leaf) must
  equal the oracle's exactly, the lists as above, and the FP64 ("plain")
  potential at every point must be within 1e-7 relative (max |u - u_o| /
  max |u_o|) of the oracle's, which restates the reference step for step and
  is pinned to the reference's goldens.  The mixed form is held to 1e-7 of
  the oracle's FP64 output on the Laplace clouds.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

CASES = ["c1_uniform20k", "mix5k_seed1", "mix20k_seed0", "uniform3k_cut16",
         "annulus6k_k0", "cluster_dup", "mix2k_cut8"]


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _make(x, y, kernel, k, neq, cut, **kw):
    import pykifmm2d_b200 as P
    kern = P.LaplaceKernel() if kernel == 0 else P.ModifiedHelmholtzKernel(k)
    return P.FMM(x, y, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), neq, cut, **kw)


def _check_lists(f, nodes, coll_ref, m2l_ref, p2p_ref):
    coll, m2l, p2p = f.export_lists()
    np.testing.assert_array_equal(coll, coll_ref)
    np.testing.assert_array_equal(p2p, p2p_ref)
    fake = nodes[:, 4] == 1
    keep = ~fake[m2l_ref[:, 0]]
    np.testing.assert_array_equal(m2l, m2l_ref[keep])
    assert f.tree_info().n_m2l_pairs == m2l.shape[0]
    return m2l.shape[0], int((~keep).sum())


@pytest.mark.parametrize("name", CASES)
def test_lists_vs_reference(golden_cases, name):
    g = golden_cases[name]
    f = _make(g["x"], g["y"], int(g["kernel"]), float(g["k"]), int(g["nequiv"]), int(g["ncutoff"]))
    f.build_tree()
    nodes, _ = f.export_tree()
    np.testing.assert_array_equal(nodes, g["nodes"])
    used, into_fake = _check_lists(f, nodes, g["colleagues"], g["m2l_pairs"], g["p2p_pairs"])
    print(f"{name}: M2L pairs {used} (+{into_fake} into fake leaves in the reference), "
          f"P2P pairs {g['p2p_pairs'].shape[0]}")


FULL = ["c2", "c3", "c4"]


@pytest.mark.parametrize("cfg_name", FULL)
def test_full_size_tree_lists_and_fp64_vs_oracle(cfg_name):
    from bench import CONFIGS
    from oracle import oracle as O
    cfg = CONFIGS[cfg_name]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    f = _make(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"])
    f.build_tree()
    o = O.OracleFMM(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"])
    nodes_o, _ = o.tree.export()
    nodes_g, pl_g = f.export_tree()
    np.testing.assert_array_equal(nodes_g, nodes_o)
    np.testing.assert_array_equal(pl_g, o.tree.locate(x, y))
    used, into_fake = _check_lists(f, nodes_o, *o.tree.lists())
    f.precompute()
    f.build_expansions(tau)
    pot = f.evaluate_to_points(f.x, f.y, True)
    o.build_expansions(tau)
    po = o.evaluate_to_points(x, y, True)
    e = rel(pot, po)
    print(f"{cfg_name}: {nodes_g.shape[0]} nodes, M2L pairs {used} (+{into_fake} into fake leaves in the "
          f"reference); fp64 vs oracle at all {x.size} points {e:.2e}")
    assert e <= 1e-7


@pytest.mark.parametrize("cfg_name", ["c2", "c3"])
def test_full_size_mixed_vs_oracle(cfg_name):
    """The mixed form at full size against the oracle's FP64 output at every
    point.  With the FP64 near field (near_fp64) only the int8 tensor-core M2L
    differs from the plain form: <= 1e-7 at every point.  With the FP32 near
    field: <= 1e-7 at 99.9% of the points.  The rest have a neighbour closer
    than ~2^-10 of their leaf width (all of them on the unit circle of the 1M
    mixture, where 200k points lie on a curve and the closest pair is 2.6e-8
    leaf widths apart); FP32 offsets inside a leaf resolve 2^-24 leaf widths,
    so such pairs carry a relative error of ~2^-24 / separation in their
    logarithm."""
    from bench import CONFIGS
    from oracle import oracle as O
    cfg = CONFIGS[cfg_name]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    o = O.OracleFMM(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"])
    o.build_expansions(tau)
    po = o.evaluate_to_points(x, y, True)
    scale = np.abs(po).max()
    f = _make(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"], precision="mixed", near_fp64=True)
    f.build_expansions(tau)
    e64 = rel(f.evaluate_to_points(f.x, f.y, True), po)
    f = _make(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"], precision="mixed")
    f.build_expansions(tau)
    err = np.abs(f.evaluate_to_points(f.x, f.y, True) - po) / scale
    q = np.quantile(err, 0.999)
    print(f"{cfg_name}: int8 M2L + FP64 near field vs oracle at all {x.size} points {e64:.2e}; FP32 near field: "
          f"99.9% of points {q:.2e}, max {err.max():.2e}")
    assert e64 <= 1e-7
    assert q <= 1e-7


def test_c4_mixed_vs_oracle():
    """The K0 annulus in the mixed form (FP32 K0 near field): measured against
    the oracle's FP64 output at every point; bound 1e-6."""
    from bench import CONFIGS
    from oracle import oracle as O
    cfg = CONFIGS["c4"]
    x, y, tau = cfg["gen"](cfg["n"], 0)
    f = _make(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"], precision="mixed")
    f.build_expansions(tau)
    pot = f.evaluate_to_points(f.x, f.y, True)
    o = O.OracleFMM(x, y, cfg["kernel"], cfg["k"], cfg["neq"], cfg["cut"])
    o.build_expansions(tau)
    po = o.evaluate_to_points(x, y, True)
    e = rel(pot, po)
    print(f"c4: mixed vs oracle fp64 at all {x.size} points {e:.2e}")
    assert e <= 1e-6
