"""Failure detection through the C ABI, with no GPU fault: every failure is made on
the host (a NaN in a host-supplied input, an iteration cap, a workspace cap) or by a
device wait whose bound is set so short that it runs out, and each test checks that
the call returns its status and that the context stays usable afterwards."""
import ctypes as C

import numpy as np
import pytest
import torch

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, complex).T)).cuda()


def _gemm(ctx, A, B):
    M, K = A.shape
    N = B.shape[1]
    dA, dB = _dev(A), _dev(B)
    Cd = torch.zeros((N, M), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    st = ctx.lib.imps_zgemm(ctx.h, 0, 0, M, N, K, 1.0, 0.0, C.c_void_p(dA.data_ptr()), M,
                            C.c_void_p(dB.data_ptr()), K, 0.0, 0.0, C.c_void_p(Cd.data_ptr()), M)
    if st == L.IMPS_OK:
        ctx.synchronize()
    return st, Cd.cpu().numpy().T


def test_bounded_wait_runs_out_and_context_recovers():
    c = imps.Context(0)
    c.set_precision(L.IMPS_PREC_SPLIT_I8, 4)
    rng = np.random.default_rng(1)
    A = rng.standard_normal((512, 512)) + 1j * rng.standard_normal((512, 512))
    B = rng.standard_normal((512, 512)) + 1j * rng.standard_normal((512, 512))
    # a one-cycle bound: the first wait of the GEMM pipeline that is not already
    # satisfied gives up; the kernel drains its copies and MMAs and returns
    assert c.lib.imps_ctx_set_wait_limit(c.h, 1) == L.IMPS_OK
    st, _ = _gemm(c, A, B)
    assert st == L.IMPS_TIMEOUT
    assert b"bounded device wait" in c.lib.imps_ctx_last_error(c.h)
    # default bound again: the same context computes the product
    assert c.lib.imps_ctx_set_wait_limit(c.h, 0) == L.IMPS_OK
    st, got = _gemm(c, A, B)
    assert st == L.IMPS_OK
    assert rel(got, A @ B) < 1e-6
    c.close()


@pytest.fixture(scope="module")
def small_problem():
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    opsi = O.randomimps([2, 2], D=12, seed=31)
    return oH, opsi, O.build_envs(opsi, oH)


def _eigsolve(ctx, envs, H, x0, tol=1e-10, krylovdim=30, maxiter=300):
    x = np.zeros_like(x0)
    info = L.KrylovInfo()
    st = ctx.lib.imps_eigsolve_ac(envs.h, H.handle(ctx), 0, L.dptr(x0), L.dptr(x), tol, krylovdim, maxiter, 1,
                                  C.byref(info))
    return st, x, info


def _setup(small_problem):
    ctx = imps.Context(0)
    oH, opsi, oenvs = small_problem
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = upload_envs(psi, H, oenvs)
    return ctx, H, psi, envs


def test_nan_in_start_vector(small_problem):
    ctx, H, psi, envs = _setup(small_problem)
    opsi = small_problem[1]
    x0 = np.asfortranarray(opsi.AC[0].copy())
    x0[3, 1, 2] = np.nan
    st, _, _ = _eigsolve(ctx, envs, H, x0)
    assert st == L.IMPS_INVALID_ARG
    assert b"NaN" in ctx.lib.imps_ctx_last_error(ctx.h)
    st, x, info = _eigsolve(ctx, envs, H, np.asfortranarray(opsi.AC[0]))
    assert st == L.IMPS_OK and info.converged == 1 and np.all(np.isfinite(x))
    ctx.close()


def test_nan_in_environment(small_problem):
    ctx, H, psi, envs = _setup(small_problem)
    oH, opsi, oenvs = small_problem
    GL = np.asfortranarray(oenvs.lefts[0].copy())
    GL[0, 1, 0] = np.inf
    envs.set_leftenv(1, GL)
    st, _, _ = _eigsolve(ctx, envs, H, np.asfortranarray(opsi.AC[0]))
    assert st == L.IMPS_INVALID_ARG
    assert b"non-finite" in ctx.lib.imps_ctx_last_error(ctx.h)
    envs.set_leftenv(1, oenvs.lefts[0])
    st, _, info = _eigsolve(ctx, envs, H, np.asfortranarray(opsi.AC[0]))
    assert st == L.IMPS_OK and info.converged == 1
    ctx.close()


def test_iteration_cap_is_not_converged(small_problem):
    # the reference only warns (KrylovKit info.converged == 0): the ABI reports
    # IMPS_NOT_CONVERGED and still writes the best Ritz vector
    ctx, H, psi, envs = _setup(small_problem)
    opsi = small_problem[1]
    st, x, info = _eigsolve(ctx, envs, H, np.asfortranarray(opsi.AC[0]), tol=1e-15, krylovdim=3, maxiter=1)
    assert st == L.IMPS_NOT_CONVERGED
    assert info.converged == 0 and info.numiter == 1
    assert abs(np.linalg.norm(x) - 1) < 1e-12
    ctx.close()


def test_workspace_cap_is_oom_and_recoverable(small_problem):
    ctx, H, psi, envs = _setup(small_problem)
    oH, opsi, oenvs = small_problem
    assert ctx.lib.imps_ctx_set_workspace_limit(ctx.h, 4096) == L.IMPS_OK
    st, _, _ = _eigsolve(ctx, envs, H, np.asfortranarray(opsi.AC[0]))
    assert st == L.IMPS_OOM
    assert b"workspace limit" in ctx.lib.imps_ctx_last_error(ctx.h)
    used = C.c_int64()
    assert ctx.lib.imps_ctx_workspace_bytes(ctx.h, C.byref(used)) == L.IMPS_OK
    assert used.value <= 4096
    assert ctx.lib.imps_ctx_set_workspace_limit(ctx.h, 0) == L.IMPS_OK
    st, x, info = _eigsolve(ctx, envs, H, np.asfortranarray(opsi.AC[0]))
    assert st == L.IMPS_OK and info.converged == 1
    xr = O.lanczos_eigsolve(lambda v: O.ac_apply(oenvs.lefts[0], oH[0], oenvs.rights[0], v), opsi.AC[0], 1e-10,
                            30, 300, True)[1]
    assert rel(x, xr) < 1e-6
    ctx.close()
