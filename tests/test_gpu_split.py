"""The int8 split-precision complex GEMM (tcgen05) through the C ABI.

* Integer-valued operands with |re|, |im| <= 100 are represented exactly by the
  first slice, so the product must be bit-exact against the exact integer
  product (this pins the MMA descriptors, the TMA layout and the epilogue).
* Random operands: error bounded by the slice truncation, relative to |A||B|.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu

OPS = {"N": 0, "C": 2}


def dev(a):
    # column-major complex128 on the device: store the transpose row-major
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, complex).T)).cuda()


def host(t, shape):
    return t.cpu().numpy().T.reshape(shape)


def run_gemm(ctx, opA, opB, A, B, Cinit=None, beta=0.0):
    Am = A if opA == "N" else A.conj().T
    Bm = B if opB == "N" else B.conj().T
    M, K = Am.shape
    N = Bm.shape[1]
    dA, dB = dev(A), dev(B)
    Cd = dev(np.zeros((M, N), complex) if Cinit is None else Cinit)
    st = ctx.lib.imps_zgemm(ctx.h, OPS[opA], OPS[opB], M, N, K, 1.0, 0.0, C.c_void_p(dA.data_ptr()), A.shape[0],
                            C.c_void_p(dB.data_ptr()), B.shape[0], beta, 0.0, C.c_void_p(Cd.data_ptr()), M)
    L.check(st, ctx.h)
    return host(Cd, (M, N)), Am @ Bm


@pytest.fixture()
def split_ctx():
    c = imps.Context(0)
    c.set_precision(L.IMPS_PREC_SPLIT_I8, 2)
    yield c
    c.close()


@pytest.mark.parametrize("M,N,K", [(512, 256, 300), (300, 520, 260), (128, 1000, 300)])
@pytest.mark.parametrize("opA,opB", [("N", "N"), ("C", "N"), ("N", "C"), ("C", "C")])
def test_split_gemm_bit_exact_integers(split_ctx, M, N, K, opA, opB):
    rng = np.random.default_rng(M + N + K)
    A0 = rng.integers(-100, 101, (M, K)) + 1j * rng.integers(-100, 101, (M, K))
    B0 = rng.integers(-100, 101, (K, N)) + 1j * rng.integers(-100, 101, (K, N))
    A = A0 if opA == "N" else A0.conj().T
    B = B0 if opB == "N" else B0.conj().T
    got, ref = run_gemm(split_ctx, opA, opB, A, B)
    assert np.array_equal(got, ref), f"max diff {np.abs(got - ref).max()}"


@pytest.mark.parametrize("s", [3, 4, 5, 6])
@pytest.mark.parametrize("M,N,K", [(256, 384, 400), (64, 64, 12000)])
def test_split_gemm_bit_exact_slice_counts(s, M, N, K):
    # slice counts with 2 and 1 TMEM tile buffers and 5 to 2 pipeline stages, and a K
    # long enough to be cut into several int32-safe groups at 6 slices (sizes above the
    # split dispatch threshold M N K >= 2^25)
    c = imps.Context(0)
    try:
        c.set_precision(L.IMPS_PREC_SPLIT_I8, s)
        rng = np.random.default_rng(s * 1000 + K)
        A = rng.integers(-100, 101, (M, K)) + 1j * rng.integers(-100, 101, (M, K))
        B = rng.integers(-100, 101, (K, N)) + 1j * rng.integers(-100, 101, (K, N))
        Am, Bm = dev(A), dev(B)
        Cd = dev(np.zeros((M, N), complex))
        L.check(c.lib.imps_zgemm(c.h, 0, 0, M, N, K, 1.0, 0.0, C.c_void_p(Am.data_ptr()), M, C.c_void_p(Bm.data_ptr()),
                                 K, 0.0, 0.0, C.c_void_p(Cd.data_ptr()), M), c.h)
        assert np.array_equal(host(Cd, (M, N)), A @ B)
    finally:
        c.close()


@pytest.mark.parametrize("s", [2, 3, 4, 5, 6])
@pytest.mark.parametrize("M,N,K,opB", [(300, 200, 600, "N"), (520, 136, 700, "C"), (64, 200, 17000, "N")])
def test_split_gemm_bit_exact_wide_tiles(s, M, N, K, opB):
    # slice counts 2..4 run 128-column tiles, 5 and 6 run 96- and 80-column tiles: N
    # ragged against the tile (the last tile part valid, its B box partly past the
    # 128-row padded planes for 96 / 80 columns), and at 4..6 slices K = 17000 is cut
    # into two int32-safe groups, whose later group the epilogue adds onto the first
    # one's output
    c = imps.Context(0)
    try:
        c.set_precision(L.IMPS_PREC_SPLIT_I8, s)
        rng = np.random.default_rng(s * 7 + N + K)
        A = rng.integers(-100, 101, (M, K)) + 1j * rng.integers(-100, 101, (M, K))
        B0 = rng.integers(-100, 101, (K, N)) + 1j * rng.integers(-100, 101, (K, N))
        B = B0 if opB == "N" else B0.conj().T
        got, ref = run_gemm(c, "N", opB, A, B)
        assert np.array_equal(got, ref), f"max diff {np.abs(got - ref).max()}"
        # accumulate onto an existing C through the same tiles
        C0 = rng.integers(-9, 10, (M, N)).astype(complex)
        got2, _ = run_gemm(c, "N", opB, A, B, Cinit=C0, beta=1.0)
        assert np.array_equal(got2, ref + C0)
    finally:
        c.close()


def test_split_gemm_accumulate(split_ctx):
    rng = np.random.default_rng(7)
    A = rng.integers(-50, 51, (200, 600)) + 1j * rng.integers(-50, 51, (200, 600))
    B = rng.integers(-50, 51, (600, 300)) + 1j * rng.integers(-50, 51, (600, 300))
    C0 = rng.integers(-9, 10, (200, 300)).astype(complex)
    got, ref = run_gemm(split_ctx, "N", "N", A, B, Cinit=C0, beta=1.0)
    assert np.array_equal(got, ref + C0)


@pytest.mark.parametrize("s", [3, 4, 5, 6])
def test_split_gemm_accuracy(s):
    c = imps.Context(0)
    c.set_precision(L.IMPS_PREC_SPLIT_I8, s)
    rng = np.random.default_rng(s)
    M, N, K = 384, 512, 640
    A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    A[:7] *= 1e-6  # rows of very different magnitude: per-row scaling must keep them accurate
    got, ref = run_gemm(c, "N", "N", A, B)
    # per element: truncation of each operand below 2^-7s of its row / column scale
    # (scale < 2 x max(|re|, |im|)), summed over the 2K real products
    ra = 2 * np.maximum(np.abs(A.real), np.abs(A.imag)).max(axis=1)
    cb = 2 * np.maximum(np.abs(B.real), np.abs(B.imag)).max(axis=0)
    bound = np.outer(ra, cb) * 2 * K * (s + 2) * 2.0 ** (-7 * s)
    err = np.abs(got - ref)
    assert np.all(err <= bound), f"worst ratio {np.max(err / bound)}"
    c.close()


def test_split_heff_matches_fp64():
    # AC Heff through the split engine vs the FP64 engine on the same environments
    c64 = imps.default_context()
    cs = imps.Context(0)
    cs.set_precision(L.IMPS_PREC_SPLIT_I8, 5)
    oH = O.SchurMPO([O.hubbard_hamiltonian().Ws[0]])
    opsi = O.randomimps([4], D=128, seed=3)
    oenvs = O.build_envs(opsi, oH)
    H = to_device_mpo(oH)
    x = O.random_site_tensors([4], 128, 9)[0]
    outs = []
    for ctx in (c64, cs):
        psi = upload_state(ctx, opsi)
        envs = upload_envs(psi, H, oenvs)
        outs.append(imps.AC_hamiltonian(1, psi, H, psi, envs)(x))
    yref = O.ac_apply(oenvs.lefts[0], oH[0], oenvs.rights[0], x)
    assert rel(outs[0], yref) < 1e-12
    assert rel(outs[1], yref) < 1e-8
    cs.close()


def _vumps(ctx, H, As, maxiter, tol):
    psi0 = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
    psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=As[0].shape[0], maxiter=maxiter, tol=tol))
    return imps.expectationvalue(psi, H, envs).real, info


def test_split_vumps_matches_fp64_at_convergence():
    # gapped TFIM (h = 0.5), N = 1, D = 256: every Heff / push GEMM is large enough for
    # the split engine.  Adaptive slices (the default mixed mode) converge like FP64.
    H = imps.tfim_hamiltonian(h=0.5)
    As = imps.random_site_tensors([2], 256, 17)
    e64, i64 = _vumps(imps.default_context(), H, As, 60, 1e-9)
    cs = imps.Context(0)
    cs.set_precision(L.IMPS_PREC_SPLIT_I8, 0)
    es, isp = _vumps(cs, H, As, 60, 1e-9)
    assert i64.converged and isp.converged
    assert isp.itererr < 1e-9
    assert abs(es - e64) < 1e-9
    cs.close()


def test_split_fixed_slices_floor():
    # A fixed slice count fixes the accuracy of every split product, including the
    # environment right-hand sides: with 4 slices the Galerkin error levels off near
    # 1e-7 (the solvers' FP64 refinement cannot remove an error in the operator itself)
    # while the energy stays within 1e-8 of the FP64 result.
    H = imps.tfim_hamiltonian(h=0.5)
    As = imps.random_site_tensors([2], 256, 17)
    e64, _ = _vumps(imps.default_context(), H, As, 40, 1e-9)
    cs = imps.Context(0)
    cs.set_precision(L.IMPS_PREC_SPLIT_I8, 4)
    es, isp = _vumps(cs, H, As, 40, 1e-9)
    assert min(isp.losses) < 1e-6
    assert abs(es - e64) < 1e-7
    cs.close()
