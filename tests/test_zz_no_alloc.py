"""The allocation-free AC apply (imps_ac_apply_noalloc) through the C ABI.

Callers whose own caching allocator already holds the device memory (or who must
avoid the implicit synchronisation of cudaMalloc) use this entry point; it keeps
every intermediate in a fixed device array of the library.  Here the caller-side
buffers come from torch (the caller's allocator) and the result is compared with
the regular entry point (imps_ac_apply) on two calls in a row: the second call
uses an MPO tensor with an empty right level, so stale data left in the shared
array by the first call would show up.

This file is collected last on purpose (it runs after every other test when the
suite stops at the first failure); it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _dev(a):
    # column-major complex128 in caller-owned (torch) device memory
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).ravel(order="F"))).cuda()


def _case(seed, D, W):
    rng = np.random.default_rng(seed)
    m, d, n = W.shape[0], W.shape[1], W.shape[2]

    def rc(*s):
        return np.asfortranarray(rng.standard_normal(s) + 1j * rng.standard_normal(s))
    return rc(D, m, D), rc(D, n, D), rc(D, d, D)


def _regular(ctx, W, GL, GR, x):
    H = imps.SparseIMPO([W])
    D = x.shape[0]
    psi = imps.CanonicalIMPS(ctx, [x.shape[1]], [D])
    envs = imps.DMRGCache(psi, H, build=False)
    envs.set_leftenv(1, GL)
    envs.set_rightenv(1, GR)
    return imps.AC_hamiltonian(1, psi, H, psi, envs)(x)


def _noalloc(ctx, W, GL, GR, x):
    """Returns (y, device bytes the library took during the call)."""
    m, d, n = W.shape[0], W.shape[1], W.shape[2]
    D = x.shape[0]
    Wh = np.asfortranarray(W.astype(complex))
    gl, gr, xd = _dev(GL), _dev(GR), _dev(x)
    yd = torch.zeros_like(xd)
    # the library queues its work on the context's stream: the caller's fills and
    # copies above (torch's stream) must be complete before the call reads them
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = ctx.lib.imps_ac_apply_noalloc(ctx.h, D, d, D, m, n, Wh.ctypes.data_as(L.DP), C.c_void_p(gl.data_ptr()),
                                       C.c_void_p(gr.data_ptr()), C.c_void_p(xd.data_ptr()),
                                       C.c_void_p(yd.data_ptr()))
    L.check(st, ctx.h)
    ctx.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return yd.cpu().numpy().reshape(x.shape, order="F"), free0 - free1


def test_noalloc_matches_regular_entry_point_twice():
    ctx = imps.Context(0)
    W1 = imps.hubbard_hamiltonian().Ws[0]
    W2 = np.array(imps.heisenberg_hamiltonian().Ws[0], order="F")
    W2[:, :, 2, :] = 0.0  # right level 3 has no block: its intermediate must read as zero
    for seed, D, W in ((1, 24, W1), (2, 40, W2)):
        GL, GR, x = _case(seed, D, W)
        y_ref = _regular(ctx, W, GL, GR, x)
        y, _ = _noalloc(ctx, W, GL, GR, x)
        assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    # once its kernels are loaded, a call must leave the device's free memory where
    # it was: nothing is allocated behind the caller's back
    y, took = _noalloc(ctx, W, GL, GR, x)
    assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    assert took == 0
    ctx.close()


def test_noalloc_rejects_sizes_beyond_the_array():
    ctx = imps.Context(0)
    W = imps.hubbard_hamiltonian().Ws[0]
    D = 1024  # 16 * D*d*D * (m + n) bytes >> 64 MiB
    buf = torch.zeros(8, dtype=torch.complex128, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    Wh = np.asfortranarray(W)
    st = ctx.lib.imps_ac_apply_noalloc(ctx.h, D, 4, D, 6, 6, Wh.ctypes.data_as(L.DP), p, p, p, p)
    assert st == L.IMPS_INVALID_ARG
    assert b"scratch" in ctx.lib.imps_ctx_last_error(ctx.h)
    ctx.close()
