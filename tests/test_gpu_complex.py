"""GPU parity of the complex form: FMM(..., iscomplex=True) (class_fmm.py:174)
with the Helmholtz kernel (i/4) H0(k r) (examples/hankel.py:37-39), against
the reference's own complex output (tests/golden/helm_*.npz, made by running
the reference with that plug-in) and against the oracle's complex mode.

Tolerances: trees and lists exactly; FP64 potentials max |u - u_ref| /
max |u_ref| <= 1e-9 (the real FP64 form reaches ~1e-12 against the
reference; the complex kernel's Bessel functions come from different
libraries on the two sides: the C library's j0/y0 in the reference plug-in,
CUDA's on the GPU).
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]

HELM = ["helm_uniform6k_k2", "helm_circle4k_k10"]


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def make(x, y, kern, neq, cut, **kw):
    import pykifmm2d_b200 as P
    return P.FMM(x, y, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), neq, cut, **kw)


@pytest.mark.parametrize("name", HELM)
def test_helmholtz_tree_lists_and_potential_vs_reference(golden_cases, name):
    import pykifmm2d_b200 as P
    g = golden_cases[name]
    f = make(g["x"], g["y"], P.HelmholtzKernel(float(g["k"])), int(g["nequiv"]), int(g["ncutoff"]), iscomplex=True)
    f.build_tree()
    nodes, pl = f.export_tree()
    np.testing.assert_array_equal(nodes, g["nodes"])
    np.testing.assert_array_equal(pl, g["point_leaf"])
    coll, m2l, p2p = f.export_lists()
    np.testing.assert_array_equal(coll, g["colleagues"])
    np.testing.assert_array_equal(p2p, g["p2p_pairs"])
    keep = g["nodes"][g["m2l_pairs"][:, 0], 4] == 0
    np.testing.assert_array_equal(m2l, g["m2l_pairs"][keep])
    f.build_expansions(g["tau"])
    pot = f.evaluate_to_points(f.x, f.y, True)
    assert pot.dtype == np.complex128
    e = rel(pot, g["pot"])
    et = rel(f.evaluate_to_points(g["xt"], g["yt"], False), g["pot_targets"])
    print(f"{name}: complex fp64 vs reference {e:.2e}, at targets {et:.2e}")
    assert e <= 1e-9 and et <= 1e-9


def test_helmholtz_kernel_functions_vs_scipy():
    import pykifmm2d_b200 as P
    sp = pytest.importorskip("scipy.special")
    rng = np.random.default_rng(1)
    sx, sy, tx, ty = rng.uniform(-1, 1, 29), rng.uniform(-1, 1, 29), rng.uniform(-1, 1, 17), rng.uniform(-1, 1, 17)
    tau = rng.standard_normal(29) + 1j * rng.standard_normal(29)
    kern = P.HelmholtzKernel(7.0)
    ref = 0.25j * sp.hankel1(0, 7.0 * np.hypot(tx[:, None] - sx[None, :], ty[:, None] - sy[None, :]))
    KF, KA, KAS = P.Get_Kernel_Functions(kern)
    m = np.zeros((17, 29), dtype=complex)
    KF(sx, sy, tx, ty, m)
    np.testing.assert_allclose(m, ref, rtol=1e-12, atol=1e-13)
    a = np.zeros(17, dtype=complex)
    KA(sx, sy, tx, ty, tau, a)
    np.testing.assert_allclose(a, ref @ tau, rtol=1e-12, atol=1e-12)
    s = np.zeros(29, dtype=complex)
    KAS(sx, sy, tau, s)
    full = 0.25j * sp.hankel1(0, 7.0 * np.hypot(sx[:, None] - sx[None, :], sy[:, None] - sy[None, :]) +
                              np.eye(29))
    np.fill_diagonal(full, 0.0)
    np.testing.assert_allclose(s, full @ tau, rtol=1e-12, atol=1e-12)


def test_complex_density_with_a_real_kernel():
    """iscomplex=True with the Laplace kernel: the complex potential equals the
    real form applied to the real and imaginary parts."""
    import pykifmm2d_b200 as P
    rng = np.random.default_rng(2)
    x, y = rng.uniform(-1, 1, 30_000), rng.uniform(-1, 1, 30_000)
    tau = rng.standard_normal(x.size) + 1j * rng.standard_normal(x.size)
    kern = P.LaplaceKernel()
    fc = make(x, y, kern, 24, 50, iscomplex=True)
    fc.build_expansions(tau)
    pc = fc.evaluate_to_points(fc.x, fc.y, True)
    fr = make(x, y, kern, 24, 50)
    fr.build_expansions(tau.real)
    pr = fr.evaluate_to_points(fr.x, fr.y, True)
    fr.build_expansions(tau.imag)
    pi = fr.evaluate_to_points(fr.x, fr.y, True)
    assert rel(pc, pr + 1j * pi) <= 1e-12


def test_helmholtz_200k_vs_oracle():
    import pykifmm2d_b200 as P
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    n = 200_000
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    tau = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    f = make(x, y, P.HelmholtzKernel(5.0), 24, 64, iscomplex=True)
    f.build_expansions(tau)
    pot = f.evaluate_to_points(f.x, f.y, True)
    o = O.OracleFMM(x, y, O.KERNEL_HELMHOLTZ, 5.0, 24, 64)
    nodes_o, _ = o.tree.export()
    np.testing.assert_array_equal(f.export_tree()[0], nodes_o)
    o.build_expansions(tau)
    e = rel(pot, o.evaluate_to_points(x, y, True))
    idx = np.random.default_rng(123).choice(n, 256, replace=False)
    ed = rel(pot[idx], O.direct(x, y, tau, idx, O.KERNEL_HELMHOLTZ, 5.0))
    print(f"helmholtz 200k: complex fp64 vs oracle {e:.2e}, vs direct sum at 256 targets {ed:.2e}")
    assert e <= 1e-9
    assert ed <= 1e-5


def test_complex_form_errors():
    import pykifmm2d_b200 as P
    from pykifmm2d_b200 import _lib as B
    x = np.random.default_rng(4).uniform(-1, 1, 500)
    with pytest.raises(ValueError):
        make(x, x[::-1].copy(), P.HelmholtzKernel(2.0), 16, 20)
    with pytest.raises(B.KifmmError) as e:
        make(x, x[::-1].copy(), P.HelmholtzKernel(2.0), 16, 20, iscomplex=True, precision="mixed")
    assert e.value.code == B.ERR_UNSUPPORTED
    with pytest.raises(B.KifmmError) as e:
        make(x, x[::-1].copy(), P.HelmholtzKernel(2.0), 40, 20, iscomplex=True)
    assert e.value.code == B.ERR_ARG
