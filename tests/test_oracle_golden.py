"""Pin the C oracle against the golden vectors produced by the reference itself
(tests/golden/make_golden.py runs pykifmm2d/class_fmm.py's FMM)."""
import numpy as np
import pytest

from oracle import oracle as O

CASES = ["c1_uniform20k", "mix5k_seed1", "mix20k_seed0", "uniform3k_cut16",
         "annulus6k_k0", "cluster_dup", "mix2k_cut8", "helm_uniform6k_k2", "helm_circle4k_k10"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_tree_matches_reference(golden_cases, name):
    g = golden_cases[name]
    t = O.OracleTree(g["x"], g["y"], int(g["ncutoff"]))
    nodes, root = t.export()
    assert t.levels == int(g["levels"])
    np.testing.assert_array_equal(root, g["root"])
    np.testing.assert_array_equal(nodes, g["nodes"])
    np.testing.assert_array_equal(t.locate(g["x"], g["y"]), g["point_leaf"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_potential_matches_reference(golden_cases, name):
    g = golden_cases[name]
    f = O.OracleFMM(g["x"], g["y"], int(g["kernel"]), float(g["k"]), int(g["nequiv"]), int(g["ncutoff"]))
    f.build_expansions(g["tau"])
    pot = f.evaluate_to_points(g["x"], g["y"], True)
    # same algorithm in FP64; only summation order and the LU kernel differ
    assert np.abs(pot - g["pot"]).max() / np.abs(g["pot"]).max() < 1e-10
    if "xt" in g:
        pt = f.evaluate_to_points(g["xt"], g["yt"], False)
        assert np.abs(pt - g["pot_targets"]).max() / np.abs(g["pot_targets"]).max() < 1e-10


def test_oracle_direct_matches_reference_kas(golden_cases):
    g = golden_cases["c1_uniform20k"]
    idx = np.random.default_rng(123).choice(g["x"].size, 256, replace=False)
    d = O.direct(g["x"], g["y"], g["tau"], idx)
    np.testing.assert_allclose(d, g["direct"][idx], rtol=0, atol=1e-11 * np.abs(g["direct"]).max())


def test_oracle_k0_against_scipy():
    sp = pytest.importorskip("scipy.special")
    x = np.concatenate([np.geomspace(1e-8, 2, 200), np.linspace(2, 60, 400)])
    np.testing.assert_allclose(O.k0(x), sp.k0(x), rtol=3e-14)


def test_repeated_apply_is_fresh(golden_cases):
    """The reference accumulates into stale check potentials on a second
    build_expansions (tree.py:414 + class_fmm.py:71); the oracle zeroes them."""
    g = golden_cases["uniform3k_cut16"]
    f = O.OracleFMM(g["x"], g["y"], 0, 0.0, int(g["nequiv"]), int(g["ncutoff"]))
    f.build_expansions(g["tau"] * 3.0)
    f.build_expansions(g["tau"])
    pot = f.evaluate_to_points(g["x"], g["y"], True)
    assert np.abs(pot - g["pot"]).max() / np.abs(g["pot"]).max() < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_oracle_lists_match_reference(golden_cases, name):
    """Colleagues by direction, M2L (target, source) pairs and P2P (leaf,
    source) pairs read from the reference's own Level arrays
    (make_golden.reference_lists) equal the oracle's, exactly."""
    g = golden_cases[name]
    t = O.OracleTree(g["x"], g["y"], int(g["ncutoff"]))
    coll, m2l, p2p = t.lists()
    np.testing.assert_array_equal(coll, g["colleagues"])
    np.testing.assert_array_equal(m2l, g["m2l_pairs"])
    np.testing.assert_array_equal(p2p, g["p2p_pairs"])


@pytest.mark.parametrize("name", ["helm_uniform6k_k2", "helm_circle4k_k10"])
def test_oracle_complex_direct_matches_reference_kas(golden_cases, name):
    g = golden_cases[name]
    idx = np.random.default_rng(5).choice(g["x"].size, 200, replace=False)
    d = O.direct(g["x"], g["y"], g["tau"], idx, int(g["kernel"]), float(g["k"]))
    assert np.abs(d - g["direct"][idx]).max() <= 1e-12 * np.abs(g["direct"]).max()
