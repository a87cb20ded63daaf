"""ctypes wrapper of the C oracle (``kifmm_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker.  The product
(``pykifmm2d_b200``) never imports it.

The oracle restates the reference's ``class_fmm.FMM`` pipeline
(pykifmm2d/class_fmm.py:166-402 over pykifmm2d/tree.py:460-727) in C with
OpenMP; ``OracleFMM`` mirrors the reference's method names.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libkifmm_oracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p


def build():
    """Compile the oracle library in place (gcc + OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(_HERE, f) for f in ("kifmm_oracle.c", "kifmm_oracle_fmm.inc")]
        if not os.path.exists(_LIB) or any(os.path.getmtime(_LIB) < os.path.getmtime(f) for f in srcs):
            build()
        L = ctypes.CDLL(_LIB)
        L.ork_tree_build.argtypes = [_d, _d, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(_vp)]
        L.ork_tree_build.restype = ctypes.c_int
        L.ork_tree_levels.argtypes = [_vp]
        L.ork_tree_levels.restype = ctypes.c_int
        L.ork_tree_num_nodes.argtypes = [_vp]
        L.ork_tree_num_nodes.restype = ctypes.c_int64
        L.ork_tree_export.argtypes = [_vp, _i64, _d]
        L.ork_locate.argtypes = [_vp, _d, _d, ctypes.c_int64, _i64]
        L.ork_tree_colleagues.argtypes = [_vp, _i64]
        L.ork_m2l_pairs.argtypes = [_vp, _i64]
        L.ork_m2l_pairs.restype = ctypes.c_int64
        L.ork_p2p_pairs.argtypes = [_vp, _i64]
        L.ork_p2p_pairs.restype = ctypes.c_int64
        L.ork_tree_free.argtypes = [_vp]
        for pre in ("ork", "orkc"):  # real and complex values (complex: pointers to complex128)
            getattr(L, pre + "_fmm_create").argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                         ctypes.POINTER(_vp)]
            getattr(L, pre + "_fmm_create").restype = ctypes.c_int
            getattr(L, pre + "_fmm_apply").argtypes = [_vp, _vp]
            getattr(L, pre + "_fmm_eval").argtypes = [_vp, _d, _d, ctypes.c_int64, ctypes.c_int, _vp]
            getattr(L, pre + "_fmm_free").argtypes = [_vp]
            getattr(L, pre + "_direct").argtypes = [ctypes.c_int, ctypes.c_double, _d, _d, _vp, ctypes.c_int64,
                                                    _i64, ctypes.c_int64, _vp]
        L.ork_k0_value.argtypes = [ctypes.c_double]
        L.ork_k0_value.restype = ctypes.c_double
        L.ork_set_threads.argtypes = [ctypes.c_int]
        L.ork_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n):
    lib().ork_set_threads(int(n))


def max_threads():
    return lib().ork_max_threads()


def k0(x):
    return np.array([lib().ork_k0_value(float(v)) for v in np.ravel(x)])


class OracleTree:
    """Tree(x, y, ppl) of the reference (tree.py:464-522)."""

    def __init__(self, x, y, ppl, fix_bbox=False):
        self.x = _f64(x)
        self.y = _f64(y)
        h = _vp()
        rc = lib().ork_tree_build(_p(self.x), _p(self.y), self.x.size, int(ppl), int(fix_bbox), ctypes.byref(h))
        if rc:
            raise ValueError(f"oracle tree build failed (code {rc})")
        self.h = h
        self.levels = lib().ork_tree_levels(h)

    def export(self):
        n = lib().ork_tree_num_nodes(self.h)
        nodes = np.zeros((n, 7), dtype=np.int64)
        root = np.zeros(2)
        lib().ork_tree_export(self.h, _p(nodes, _i64), _p(root))
        order = np.lexsort((nodes[:, 2], nodes[:, 1], nodes[:, 0]))
        return nodes[order], root

    def lists(self):
        """Interaction lists as canonical rows of ``export()``'s node table:
        colleagues [n_nodes, 9] by direction (dx+1)*3+(dy+1) (-1: none), and
        the M2L (target, source) and P2P (leaf, source) pairs, each sorted
        (tree.py:349-375; class_fmm.py:17-33, :90-111, :323-343)."""
        n = lib().ork_tree_num_nodes(self.h)
        nodes = np.zeros((n, 7), dtype=np.int64)
        lib().ork_tree_export(self.h, _p(nodes, _i64), _p(np.zeros(2)))
        order = np.lexsort((nodes[:, 2], nodes[:, 1], nodes[:, 0]))
        rank = np.empty_like(order)
        rank[order] = np.arange(n)
        coll = np.zeros((n, 9), dtype=np.int64)
        lib().ork_tree_colleagues(self.h, _p(coll, _i64))
        coll = np.where(coll >= 0, rank[np.maximum(coll, 0)], -1)
        out_coll = np.empty_like(coll)
        out_coll[rank] = coll
        res = [out_coll]
        for f in (lib().ork_m2l_pairs, lib().ork_p2p_pairs):
            m = f(self.h, ctypes.cast(None, _i64))
            pr = np.zeros((m, 2), dtype=np.int64)
            f(self.h, _p(pr, _i64))
            pr = rank[pr]
            res.append(pr[np.lexsort((pr[:, 1], pr[:, 0]))])
        return tuple(res)

    def locate(self, x, y):
        x = _f64(x)
        y = _f64(y)
        out = np.zeros((x.size, 3), dtype=np.int64)
        lib().ork_locate(self.h, _p(x), _p(y), x.size, _p(out, _i64))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().ork_tree_free(self.h)
            self.h = None


KERNEL_LAPLACE = 0
KERNEL_K0 = 1
KERNEL_HELMHOLTZ = 2  # (i/4) H0(k r), complex


class OracleFMM:
    """Mirror of the reference's FMM (class_fmm.py:166-402) on the C oracle.
    iscomplex (class_fmm.py:174) runs it on complex values, as the Helmholtz
    kernel requires."""

    def __init__(self, x, y, kernel=KERNEL_LAPLACE, k=0.0, Nequiv=48, Ncutoff=50, fix_bbox=False, iscomplex=False):
        self.tree = OracleTree(x, y, Ncutoff, fix_bbox)
        self.iscomplex = bool(iscomplex) or kernel == KERNEL_HELMHOLTZ
        self.dtype = np.complex128 if self.iscomplex else np.float64
        self._pre = "orkc" if self.iscomplex else "ork"
        h = _vp()
        rc = getattr(lib(), self._pre + "_fmm_create")(self.tree.h, int(kernel), float(k), int(Nequiv),
                                                       ctypes.byref(h))
        if rc:
            raise ValueError(f"oracle precompute failed (code {rc})")
        self.h = h

    def build_expansions(self, tau):
        self.tau = np.ascontiguousarray(tau, dtype=self.dtype)
        getattr(lib(), self._pre + "_fmm_apply")(self.h, self.tau.ctypes.data)

    def evaluate_to_points(self, x, y, check_self=False):
        x = _f64(x)
        y = _f64(y)
        pot = np.zeros(x.size, dtype=self.dtype)
        getattr(lib(), self._pre + "_fmm_eval")(self.h, _p(x), _p(y), x.size, int(bool(check_self)), pot.ctypes.data)
        return pot

    def __del__(self):
        if getattr(self, "h", None):
            getattr(lib(), self._pre + "_fmm_free")(self.h)
            self.h = None


def direct(x, y, tau, targets, kernel=KERNEL_LAPLACE, k=0.0):
    """FP64 direct sum at selected targets, skipping only i == j (the KAS of
    class_fmm.py:134-143); complex for complex charges or the Helmholtz kernel."""
    x, y = _f64(x), _f64(y)
    cplx = np.iscomplexobj(tau) or kernel == KERNEL_HELMHOLTZ
    tau = np.ascontiguousarray(tau, dtype=np.complex128 if cplx else np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros(t.size, dtype=tau.dtype)
    getattr(lib(), "orkc_direct" if cplx else "ork_direct")(int(kernel), float(k), _p(x), _p(y), tau.ctypes.data,
                                                            x.size, _p(t, _i64), t.size, out.ctypes.data)
    return out
