"""Device densities for serving (csrc/draws.cu): Philox4x32-10 + Box-Muller.

The numpy restatement below is checked on CPU against the known-answer
vectors published with the Random123 library for philox4x32 with 10 rounds;
on the GPU, ``kifmm_fill_normal`` is compared with it (1e-13 relative: the
device takes log/sqrt/sincospi from CUDA's math library, numpy from libm)."""
import ctypes

import numpy as np
import pytest

from conftest import has_gpu

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(c, k):
    c = [int(v) & MASK for v in c]
    k0, k1 = int(k[0]) & MASK, int(k[1]) & MASK
    for _ in range(10):
        p0, p1 = M0 * c[0], M1 * c[2]
        hi0, lo0, hi1, lo1 = p0 >> 32, p0 & MASK, p1 >> 32, p1 & MASK
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0, k1 = (k0 + W0) & MASK, (k1 + W1) & MASK
    return c


def normals(n, seed, index):
    out = np.empty(n)
    for j in range((n + 1) // 2):
        r = philox4x32_10([j & MASK, j >> 32, index & MASK, index >> 32], [seed & MASK, seed >> 32])
        u1 = ((((r[0] << 32) | r[1]) >> 11) + 1) * 2.0 ** -53
        u2 = ((((r[2] << 32) | r[3]) >> 11) + 1) * 2.0 ** -53
        rad = np.sqrt(-2.0 * np.log(u1))
        out[2 * j] = rad * np.cos(2 * np.pi * u2)
        if 2 * j + 1 < n:
            out[2 * j + 1] = rad * np.sin(2 * np.pi * u2)
    return out


def test_philox_known_answers():
    assert philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert philox4x32_10([MASK] * 4, [MASK, MASK]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")
def test_fill_normal_matches_restatement():
    import torch

    from pykifmm2d_b200 import _lib as B
    lib = B.load()
    for n, seed, index in [(1001, 1000, 0), (64, 1 << 40, 7), (1, 3, (1 << 33) + 5)]:
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        B.check(lib.kifmm_fill_normal(out.data_ptr(), n, seed, index, ctypes.c_void_p(1)))
        torch.cuda.synchronize()
        ref = normals(n, seed, index)
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    bad = lib.kifmm_fill_normal(out.data_ptr(), 1, (1 << 64) - 1, 0, ctypes.c_void_p(1))
    assert bad == B.ERR_ARG
