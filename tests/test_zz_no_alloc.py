"""GPU test of kifmm_morton_sort_noalloc, the entry point for callers that
cannot allocate device memory (a host that owns all device memory through
its own pool, or a loop that must not enter the allocator).

It calls the entry point through the C ABI twice in a row and checks both
outputs against the tree of the existing entry point kifmm_build_tree (its
root box from kifmm_get_tree_info, the leaf of every point from
kifmm_export_tree): integer outputs, so the comparison is exact.  The file is
named to run last, after the other tests, and also passes on its own.
"""
import ctypes

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]


def morton_np(ix, iy):
    k = np.zeros(ix.shape, dtype=np.uint64)
    for b in range(30):
        k |= ((ix.astype(np.uint64) >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b + 1)
        k |= ((iy.astype(np.uint64) >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b)
    return k


def test_noalloc_sort_matches_tree_build():
    import torch

    import pykifmm2d_b200 as P
    from bench import gen_mixture
    from pykifmm2d_b200 import _lib as B

    x, y, _ = gen_mixture(300_000, 2)
    n = x.size
    kern = P.LaplaceKernel()
    f = P.FMM(x, y, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), 32, 64)
    f.build_tree()
    info = f.tree_info()
    _, point_leaf = f.export_tree()

    lib = B.load()
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y).cuda()
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    for call in range(2):
        keys.fill_(-1)
        perm.fill_(-1)
        torch.cuda.synchronize()
        rc = lib.kifmm_morton_sort_noalloc(xd.data_ptr(), yd.data_ptr(), n, info.root_min, info.root_max,
                                           keys.data_ptr(), perm.data_ptr(), None)
        torch.cuda.synchronize()
        B.check(rc)
        k = keys.cpu().numpy().view(np.uint64)
        p = perm.cpu().numpy().astype(np.int64)
        assert np.all(k[1:] >= k[:-1]), f"call {call}: keys not sorted"
        assert np.array_equal(np.sort(p), np.arange(n)), f"call {call}: perm is not a permutation"
        eq = k[1:] == k[:-1]
        assert np.all(p[1:][eq] > p[:-1][eq]), f"call {call}: sort not stable"
        # each key's prefix at its leaf's level is that leaf's cell in the existing tree
        lev = point_leaf[p, 0].astype(np.uint64)
        prefix = k >> (np.uint64(2) * (np.uint64(29) - lev))
        assert np.array_equal(prefix, morton_np(point_leaf[p, 1], point_leaf[p, 2])), f"call {call}: leaf mismatch"


def test_noalloc_sort_rejects_too_many_points():
    import torch

    from pykifmm2d_b200 import _lib as B
    lib = B.load()
    n = B.NOALLOC_MAX_POINTS + 1
    buf = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.kifmm_morton_sort_noalloc(buf.data_ptr(), buf.data_ptr(), n, -1.0, 1.0, buf.data_ptr(),
                                       buf.data_ptr(), None)
    assert rc == B.ERR_ARG
    assert "KIFMM_NOALLOC_MAX_POINTS" in lib.kifmm_last_error().decode()


def _host_keys(x, y, m, M):
    """Exact Morton keys on the host: the cell index is the number of grid
    lines m + j h (h = (M - m) / 2^29) that the coordinate is strictly above,
    clamped to the grid (the tree's strict '>' midline rule)."""
    h = np.ldexp(M - m, -29)
    top = (1 << 29) - 1

    def cell(v):
        j = np.clip(np.ceil((v - m) / h) - 1.0, 0, top).astype(np.int64)
        for _ in range(4):
            up = (j < top) & (v > m + (j + 1).astype(np.float64) * h)
            j = j + up
            dn = (j > 0) & ~(v > m + j.astype(np.float64) * h)
            j = j - dn
        return j

    return morton_np(cell(x), cell(y))


def test_noalloc_sort_at_capacity_allocates_nothing():
    """n = KIFMM_NOALLOC_MAX_POINTS exactly (the scratch offsets and the
    histogram table full): keys equal the host's exact keys in sorted order,
    perm is a stable permutation, and after a first call the device's free
    memory is the same before and after a second call."""
    import torch

    from pykifmm2d_b200 import _lib as B
    lib = B.load()
    n = B.NOALLOC_MAX_POINTS
    rng = np.random.default_rng(11)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    want = _host_keys(x, y, -1.0, 1.0)
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y).cuda()
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    free = []
    for call in range(2):
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        rc = lib.kifmm_morton_sort_noalloc(xd.data_ptr(), yd.data_ptr(), n, -1.0, 1.0, keys.data_ptr(),
                                           perm.data_ptr(), None)
        torch.cuda.synchronize()
        B.check(rc)
        k = keys.cpu().numpy().view(np.uint64)
        p = perm.cpu().numpy().astype(np.int64)
        assert np.array_equal(np.sort(p), np.arange(n)), f"call {call}: perm is not a permutation"
        assert np.array_equal(k, want[p]), f"call {call}: keys differ from the exact host keys"
        assert np.all(k[1:] >= k[:-1]), f"call {call}: keys not sorted"
        eq = k[1:] == k[:-1]
        assert np.all(p[1:][eq] > p[:-1][eq]), f"call {call}: sort not stable"
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free[1], "the second call changed the device's free memory"
