"""The FMM class and kernel plug-ins, with the reference's interface.

Mirrors dbstein/pykifmm2d ``pykifmm2d/class_fmm.py``:

* ``Get_Kernel_Functions(Kernel_Eval) -> (KF, KA, KAS)`` (class_fmm.py:115-145)
* ``prepare_numba_functions_on_the_fly(Kernel_Eval)`` (class_fmm.py:55-113)
* ``Kernel_Form(KF, sx, sy, tx=None, ty=None, out=None, mdtype=float)`` (:147-164)
* ``FMM(x, y, kernel_functions, numba_functions, Nequiv=48, Ncutoff=50,
  iscomplex=False, verbose=False)`` with ``build_tree``, ``precompute``,
  ``build_expansions``, ``evaluate_to_points``, ``evaluate_to_point``
  (class_fmm.py:166-402).

The reference JIT-specialises its loops on a user numba scalar kernel.  Here
the plug-in is a descriptor (``LaplaceKernel()``, ``ModifiedHelmholtzKernel(k)``)
naming one of the kernels compiled into the CUDA library; any other callable
is rejected with a TypeError.  All arithmetic runs on the GPU through the C
ABI of ``libkifmm2d.so``; nothing here computes potentials on the host.

Arrays: numpy float64 arrays (host) or CUDA float64 torch tensors (device).
Results come back in the same kind of array as the coordinates.
"""
import time

import numpy as np

from . import _lib as B

__all__ = ["LaplaceKernel", "ModifiedHelmholtzKernel", "HelmholtzKernel", "Get_Kernel_Functions",
           "prepare_numba_functions_on_the_fly", "Kernel_Form", "FMM", "get_level_information"]


class LaplaceKernel:
    """G(s -> t) = -log(|t - s|^2) / (4 pi) = -log|t - s| / (2 pi)
    (the reference's Laplace plug-in, examples/laplace2.py:31-36)."""

    kind = B.KERNEL_LAPLACE
    k = 0.0

    def desc(self):
        return B.KernelDesc(self.kind, 0, 0.0)

    def __call__(self, sx, sy, tx, ty):
        return -0.25 / np.pi * np.log((tx - sx) ** 2 + (ty - sy) ** 2)

    def __repr__(self):
        return "LaplaceKernel()"


class ModifiedHelmholtzKernel:
    """G(s -> t) = K0(k |t - s|) / (2 pi) (the reference's modified Helmholtz
    plug-in, examples/modified_helmholtz.py:38-43)."""

    kind = B.KERNEL_MOD_HELMHOLTZ

    def __init__(self, k):
        if not k > 0:
            raise ValueError("modified Helmholtz needs k > 0")
        self.k = float(k)

    def desc(self):
        return B.KernelDesc(self.kind, 0, self.k)

    def __call__(self, sx, sy, tx, ty):
        sx, sy, tx, ty = (np.atleast_1d(np.asarray(v, dtype=np.float64)) for v in (sx, sy, tx, ty))
        out = np.zeros((tx.size, sx.size))
        B.check(_kernel_matrix(self, sx, sy, tx, ty, out))
        return out if out.size != 1 else float(out[0, 0])

    def __repr__(self):
        return f"ModifiedHelmholtzKernel(k={self.k})"


class HelmholtzKernel:
    """G(s -> t) = (i/4) H0^(1)(k |t - s|), complex (the reference's Helmholtz
    plug-in, examples/hankel.py:37-39, used with FMM(..., iscomplex=True))."""

    kind = B.KERNEL_HELMHOLTZ
    complex_valued = True

    def __init__(self, k):
        if not k > 0:
            raise ValueError("Helmholtz needs k > 0")
        self.k = float(k)

    def desc(self):
        return B.KernelDesc(self.kind, 0, self.k)

    def __call__(self, sx, sy, tx, ty):
        sx, sy, tx, ty = (np.atleast_1d(np.asarray(v, dtype=np.float64)) for v in (sx, sy, tx, ty))
        out = np.zeros((tx.size, sx.size), dtype=np.complex128)
        B.check(_kernel_matrix(self, sx, sy, tx, ty, out))
        return out if out.size != 1 else complex(out[0, 0])

    def __repr__(self):
        return f"HelmholtzKernel(k={self.k})"


def _as_kernel(kernel):
    if isinstance(kernel, (LaplaceKernel, ModifiedHelmholtzKernel, HelmholtzKernel)):
        return kernel
    raise TypeError("kernel plug-ins are descriptors of the kernels compiled into the CUDA library: "
                    "use LaplaceKernel(), ModifiedHelmholtzKernel(k) or HelmholtzKernel(k); arbitrary numba "
                    "scalar kernels are not JIT-compiled by this implementation")


def _complex_kernel(kern):
    return getattr(kern, "complex_valued", False)


# ------------------------------------------------------------------ arrays
def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _hp(a, cplx=False):
    """(pointer, mem flag, keep-alive) of a host numpy array or torch tensor;
    cplx: complex128 values (interleaved doubles)."""
    if _is_torch(a):
        import torch
        t = a.detach()
        want = torch.complex128 if cplx else torch.float64
        if t.dtype != want:
            t = t.to(want)
        t = t.contiguous()
        return t.data_ptr(), (B.MEM_DEVICE if t.is_cuda else B.MEM_HOST), t
    arr = np.ascontiguousarray(a, dtype=np.complex128 if cplx else np.float64)
    return arr.ctypes.data, B.MEM_HOST, arr


def _numel(a):
    return a.numel() if _is_torch(a) else a.size


def _kernel_matrix(kern, sx, sy, tx, ty, out):
    return B.load().kifmm_kernel_matrix(kern.desc(), sx.ctypes.data, sy.ctypes.data, sx.size, tx.ctypes.data,
                                        ty.ctypes.data, tx.size, out.ctypes.data, B.MEM_HOST, 0)


# -------------------------------------------------------- kernel functions
def Get_Kernel_Functions(Kernel_Eval):
    """(KF, KA, KAS) of the reference (class_fmm.py:115-145), on the GPU in FP64.

    KF(sx, sy, tx, ty, out):       out[j, i] = G(s_i -> t_j)
    KA(sx, sy, tx, ty, tau, out):  out[j] = sum_i G(s_i -> t_j) tau_i
    KAS(sx, sy, tau, out):         out[j] = sum_{i != j} G(s_i -> s_j) tau_i
    """
    kern = _as_kernel(Kernel_Eval)
    lib = B.load()
    vt = np.complex128 if _complex_kernel(kern) else np.float64  # value type of the kernel

    def KF(sx, sy, tx, ty, out):
        sx, sy, tx, ty = (np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, tx, ty))
        buf = np.empty((tx.size, sx.size), dtype=vt)
        B.check(_kernel_matrix(kern, sx, sy, tx, ty, buf))
        out[...] = buf

    def KA(sx, sy, tx, ty, tau, out):
        sx, sy, tx, ty = (np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, tx, ty))
        tau = np.ascontiguousarray(tau, dtype=vt)
        buf = np.empty(tx.size, dtype=vt)
        B.check(lib.kifmm_kernel_apply(kern.desc(), sx.ctypes.data, sy.ctypes.data, sx.size, tx.ctypes.data,
                                       ty.ctypes.data, tx.size, tau.ctypes.data, buf.ctypes.data, B.MEM_HOST, 0))
        out[...] = buf

    def KAS(sx, sy, tau, out, targets=None):
        sx, sy = (np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy))
        tau = np.ascontiguousarray(tau, dtype=vt)
        tg = np.arange(sx.size, dtype=np.int64) if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
        buf = np.empty(tg.size, dtype=vt)
        B.check(lib.kifmm_direct_sum(kern.desc(), sx.ctypes.data, sy.ctypes.data, tau.ctypes.data, sx.size,
                                     tg.ctypes.data, tg.size, buf.ctypes.data, B.MEM_HOST, 0))
        out[...] = buf

    KF.kernel = KA.kernel = KAS.kernel = kern
    return KF, KA, KAS


def prepare_numba_functions_on_the_fly(Kernel_Eval):
    """Counterpart of class_fmm.py:55-113.  The reference returns its three
    JIT-specialised loops (upward pass, local evaluation, neighbour
    evaluation); here those loops are the library's CUDA kernels, so the
    returned tuple only names the kernel they are specialised on."""
    kern = _as_kernel(Kernel_Eval)
    return ("upwards_pass", kern), ("local_expansion_evaluation", kern), ("neighbor_evaluation", kern)


def Kernel_Form(KF, sx, sy, tx=None, ty=None, out=None, mdtype=float):
    """Dense kernel matrix with a zero diagonal for self interaction
    (class_fmm.py:147-164)."""
    if tx is None or ty is None:
        tx, ty, isself = sx, sy, True
    else:
        isself = sx is tx and sy is ty
    if out is None:
        out = np.empty((np.size(tx), np.size(sx)), dtype=mdtype)
    KF(sx, sy, tx, ty, out)
    if isself:
        np.fill_diagonal(out, 0.0)
    return out


def get_level_information(node_width, theta, radii="reference"):
    """Equivalent (small) and check (large) circles of a box (class_fmm.py:35-45)."""
    if radii == "reference":
        dd = 0.01
        r1 = 0.5 * node_width * (np.sqrt(2) + dd)
        r2 = 0.5 * node_width * (4 - np.sqrt(2) - 2 * dd)
    else:
        r1, r2 = 0.75 * node_width, 1.25 * node_width
    return r1 * np.cos(theta), r1 * np.sin(theta), r2 * np.cos(theta), r2 * np.sin(theta), r1, r2


_PREC = {"fp64": B.PREC_FP64, "plain": B.PREC_FP64, "mixed": B.PREC_MIXED}
_M2L = {"auto": B.M2L_AUTO, "fp32": B.M2L_FP32, "bf16x3": B.M2L_BF16X3, "fp16x3": B.M2L_FP16X3,
        "fp64": B.M2L_FP64, "int8": B.M2L_INT8, "int8x4": B.M2L_INT8X4}


class FMM(object):
    """Adaptive 2D KIFMM on one GPU with the reference's interface
    (class_fmm.py:166-402).

    Extra keyword options (defaults reproduce the reference):
      precision  'fp64' (every pass in FP64) or 'mixed' (FP32 near field,
                 compensated M2L); m2l selects the mixed M2L form;
      fix_bbox   False keeps the reference's root box (tree.py:475-484);
      radii      'reference' or '1.5/2.5';
      near_fp64  with precision='mixed', keep P2M/L2P/P2P in FP64;
      planned    keep the P2M, L2P and near-field kernel values in device
                 memory after the first apply and apply them as matrices (the
                 reference's fmm_planner / planned_fmm, fmm.py:530-814): for
                 repeated densities on one tree, evaluated at the sources;
      e2c        'dense' (Gauss-Jordan inverse of E2C, the reference's LU,
                 class_fmm.py:213-217) or 'circulant' (inverse from the DFT
                 of E2C's first row, the reference's FFT solve,
                 svd_fmm.py:239-242, :281-290);
      device, stream   CUDA device ordinal and stream handle.
    Unlike the reference, repeated ``build_expansions`` calls on one object
    are exact (workspaces are zeroed on every apply).
    """

    def __init__(self, x, y, kernel_functions, numba_functions, Nequiv=48, Ncutoff=50, iscomplex=False,
                 verbose=False, precision="fp64", m2l="auto", fix_bbox=False, radii="reference", device=None,
                 stream=None, near_fp64=False, e2c="dense", planned=False):
        kern = None
        for f in tuple(kernel_functions) + tuple(numba_functions):
            k = getattr(f, "kernel", None) if callable(f) else (f[1] if isinstance(f, tuple) else None)
            if k is not None:
                _as_kernel(k)
                if kern is not None and (k.kind != kern.kind or k.k != kern.k):
                    raise ValueError("kernel_functions and numba_functions name different kernels")
                kern = k
        if kern is None:
            raise TypeError("kernel_functions / numba_functions must come from Get_Kernel_Functions and "
                            "prepare_numba_functions_on_the_fly of this package")
        self.x = x
        self.y = y
        self.Nequiv = int(Nequiv)
        self.Ncutoff = int(Ncutoff)
        self.kernel_functions = kernel_functions
        self.numba_functions = numba_functions
        self.kernel = kern
        if _complex_kernel(kern) and not iscomplex:
            raise ValueError(f"{kern!r} has complex values: construct the FMM with iscomplex=True")
        self.iscomplex = bool(iscomplex)
        self.dtype = np.complex128 if self.iscomplex else np.float64
        self.verbose = verbose
        self.precision = precision
        self._on_device = _is_torch(x) and x.is_cuda
        opts = B.Options()
        lib = B.load()
        lib.kifmm_default_options(ctypes_byref(opts))
        opts.precision = _PREC[precision]
        opts.m2l = _M2L[m2l]
        opts.fix_bbox = int(bool(fix_bbox))
        opts.radii = 0 if radii == "reference" else 1
        opts.near_fp64 = int(bool(near_fp64))
        if e2c not in ("dense", "circulant"):
            raise ValueError("e2c must be 'dense' or 'circulant'")
        opts.e2c = B.E2C_CIRCULANT if e2c == "circulant" else B.E2C_DENSE
        opts.iscomplex = int(self.iscomplex)
        opts.planned = int(bool(planned))
        if device is None:
            device = x.device.index if self._on_device and x.device.index is not None else 0
        opts.device = int(device)
        if stream is None and self._on_device:
            import torch
            stream = torch.cuda.current_stream(x.device).cuda_stream
            if stream == 0:
                stream = 1  # torch's default stream is the legacy stream (cudaStreamLegacy)
        opts.stream = stream
        h = B.ctypes.c_void_p()
        B.check(lib.kifmm_plan_create(kern.desc(), self.Nequiv, self.Ncutoff, ctypes_byref(opts), ctypes_byref(h)))
        self._plan = h
        self._lib = lib
        self._have_tree = self._have_ops = False

    def _print(self, *a):
        if self.verbose:
            print(*a, flush=True)

    def build_tree(self):
        st = time.time()
        px, mx, kx = _hp(self.x)
        py, my, ky = _hp(self.y)
        if _numel(kx) != _numel(ky):
            raise ValueError("x and y must have the same size")
        B.check(self._lib.kifmm_build_tree(self._plan, px, py, _numel(kx), mx))
        self.N = _numel(kx)
        self._have_tree, self._have_ops = True, False
        self._print('....Tree formed in:             {:0.1f}'.format((time.time() - st) * 1000))

    def tree_info(self):
        info = B.TreeInfo()
        B.check(self._lib.kifmm_get_tree_info(self._plan, ctypes_byref(info)))
        return info

    def export_tree(self):
        """Canonical tree (level, ix, iy, leaf, fake_leaf, Xlist, ns) sorted by
        (level, ix, iy), and the leaf cell of every point."""
        info = self.tree_info()
        nodes = np.zeros((info.n_nodes, 7), dtype=np.int64)
        pl = np.zeros((self.N, 3), dtype=np.int64)
        B.check(self._lib.kifmm_export_tree(self._plan, nodes.ctypes.data, pl.ctypes.data))
        order = np.lexsort((nodes[:, 2], nodes[:, 1], nodes[:, 0]))
        return nodes[order], pl

    def export_lists(self):
        """Interaction lists as canonical rows of ``export_tree()``'s node table
        (sorted by (level, ix, iy)): colleagues [n_nodes, 9] by direction
        (dx+1)*3+(dy+1) (-1: none), then the M2L (target, source) and P2P
        (leaf, source) node pairs of the apply, each sorted."""
        info = self.tree_info()
        n = info.n_nodes
        nodes = np.zeros((n, 7), dtype=np.int64)
        B.check(self._lib.kifmm_export_tree(self._plan, nodes.ctypes.data, None))
        order = np.lexsort((nodes[:, 2], nodes[:, 1], nodes[:, 0]))
        rank = np.empty_like(order)
        rank[order] = np.arange(n)
        nm, npp = B.ctypes.c_int64(0), B.ctypes.c_int64(0)
        B.check(self._lib.kifmm_export_lists(self._plan, None, None, ctypes_byref(nm), None, ctypes_byref(npp)))
        coll = np.zeros((n, 9), dtype=np.int64)
        m2l = np.zeros((nm.value, 2), dtype=np.int64)
        p2p = np.zeros((npp.value, 2), dtype=np.int64)
        B.check(self._lib.kifmm_export_lists(self._plan, coll.ctypes.data, m2l.ctypes.data, ctypes_byref(nm),
                                             p2p.ctypes.data, ctypes_byref(npp)))
        coll = np.where(coll >= 0, rank[np.maximum(coll, 0)], -1)
        out = np.empty_like(coll)
        out[rank] = coll
        m2l, p2p = rank[m2l], rank[p2p]
        return (out, m2l[np.lexsort((m2l[:, 1], m2l[:, 0]))], p2p[np.lexsort((p2p[:, 1], p2p[:, 0]))])

    def precompute(self):
        if not self._have_tree:
            self.build_tree()
        st = time.time()
        B.check(self._lib.kifmm_precompute(self._plan))
        self._have_ops = True
        self._print('....Time for precomputations:   {:0.2f}'.format(1000 * (time.time() - st)))

    def build_expansions(self, tau):
        if not self._have_ops:
            self.precompute()
        st = time.time()
        p, m, keep = _hp(tau, self.iscomplex)
        if _numel(keep) != self.N:
            raise ValueError("tau must have one value per source point")
        self.tau = tau
        B.check(self._lib.kifmm_build_expansions(self._plan, p, m))
        self._print('....Time for expansions:        {:0.2f}'.format(1000 * (time.time() - st)))

    def _out(self, n, like, out):
        if out is not None:
            return out
        if _is_torch(like) and like.is_cuda:
            import torch
            return torch.empty(n, dtype=torch.complex128 if self.iscomplex else torch.float64, device=like.device)
        return np.empty(n, dtype=self.dtype)

    def evaluate_to_points(self, x, y, check_self=False, out=None):
        """Potential at (x, y): L2P from the leaf's local expansion plus P2P
        from the leaf's colleagues; check_self skips pairs with equal
        coordinates (class_fmm.py:379-399)."""
        px, mx, kx = _hp(x)
        py, my, ky = _hp(y)
        n = _numel(kx)
        res = self._out(n, x, out)
        pr, mr, kr = _hp(res, self.iscomplex)
        same = (x is self.x and y is self.y)
        if same:
            B.check(self._lib.kifmm_evaluate_to_sources(self._plan, pr, int(bool(check_self)), mr))
        else:
            B.check(self._lib.kifmm_evaluate_to_points(self._plan, px, py, n, int(bool(check_self)), pr, mr))
        if kr is not res and hasattr(res, "copy_"):
            res.copy_(kr)
        return res

    def evaluate_to_point(self, x, y):
        """Potential at a single point (class_fmm.py:353-378)."""
        return self.evaluate_to_points(np.array([float(x)]), np.array([float(y)]), False)

    def synchronize(self):
        B.check(self._lib.kifmm_synchronize(self._plan))

    def capture_apply(self, tau_dev, pot_dev, check_self=True):
        """Planned repeated evaluation at the sources (the reference's
        build_expansions(tau) + evaluate_to_points(x, y, check_self) per density,
        class_fmm.py:299-399) as a CUDA graph: runs the pair once from the CUDA
        tensor tau_dev into pot_dev, then keeps it captured; ``replay`` runs it
        again on whatever tau_dev holds.  Needs a plan on a created stream."""
        if not self._have_ops:
            self.precompute()
        import torch
        want = torch.complex128 if self.iscomplex else torch.float64
        for t in (tau_dev, pot_dev):
            if not (_is_torch(t) and t.is_cuda and t.dtype == want and t.is_contiguous()):
                raise ValueError(f"capture_apply needs contiguous {want} CUDA tensors (the graph keeps their addresses)")
        p_t, p_o = tau_dev.data_ptr(), pot_dev.data_ptr()
        if _numel(tau_dev) != self.N or _numel(pot_dev) != self.N:
            raise ValueError("tau_dev and pot_dev must have one value per source point")
        B.check(self._lib.kifmm_graph_capture(self._plan, p_t, p_o, int(bool(check_self))))

    def replay(self):
        """One graph launch of the captured apply (asynchronous on the plan's stream)."""
        B.check(self._lib.kifmm_graph_launch(self._plan))

    def __del__(self):
        h = getattr(self, "_plan", None)
        if h is not None and h.value:
            self._lib.kifmm_plan_destroy(h)
            self._plan = None


def ctypes_byref(o):
    return B.ctypes.byref(o)
