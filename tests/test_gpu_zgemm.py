"""The FP64 complex GEMM engines (DMMA tensor-core kernel, and the SIMT DFMA
kernel kept beside it) through the C ABI: every op pair, ragged shapes, complex
alpha and beta.  Integer-valued inputs are exact in FP64, so those products
must be bit-exact; random inputs agree with NumPy to 1e-13 relative."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L

pytestmark = pytest.mark.gpu
OPS = {"N": 0, "T": 1, "C": 2}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, complex).T)).cuda()


def host(t, shape):
    return t.cpu().numpy().T.reshape(shape)


def opm(X, op):
    return X if op == "N" else (X.T if op == "T" else X.conj().T)


@pytest.fixture(scope="module", params=["dmma", "simt"])
def engine_ctx(request):
    old = os.environ.get("IMPS_FP64_ENGINE")
    os.environ["IMPS_FP64_ENGINE"] = "1" if request.param == "simt" else "0"
    c = imps.Context(0)
    if old is None:
        del os.environ["IMPS_FP64_ENGINE"]
    else:
        os.environ["IMPS_FP64_ENGINE"] = old
    yield c
    c.close()


def gemm(ctx, opA, opB, A, B, alpha, beta, C0):
    M, N = C0.shape
    K = opm(A, opA).shape[1]
    dA, dB, dC = dev(A), dev(B), dev(C0)
    L.check(ctx.lib.imps_zgemm(ctx.h, OPS[opA], OPS[opB], M, N, K, alpha.real, alpha.imag, C.c_void_p(dA.data_ptr()),
                               A.shape[0], C.c_void_p(dB.data_ptr()), B.shape[0], beta.real, beta.imag,
                               C.c_void_p(dC.data_ptr()), M), ctx.h)
    return host(dC, (M, N))


@pytest.mark.parametrize("opA", ["N", "T", "C"])
@pytest.mark.parametrize("opB", ["N", "T", "C"])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (7, 130, 9), (129, 65, 17), (300, 70, 1000)])
def test_integer_products_bit_exact(engine_ctx, opA, opB, M, N, K):
    rng = np.random.default_rng(M * 31 + N * 7 + K)
    Am = rng.integers(-40, 41, (M, K)) + 1j * rng.integers(-40, 41, (M, K))
    Bm = rng.integers(-40, 41, (K, N)) + 1j * rng.integers(-40, 41, (K, N))
    A = opm(Am, opA) if opA == "N" else (Am.T if opA == "T" else Am.conj().T)
    B = opm(Bm, opB) if opB == "N" else (Bm.T if opB == "T" else Bm.conj().T)
    C0 = (rng.integers(-5, 6, (M, N)) + 1j * rng.integers(-5, 6, (M, N))).astype(complex)
    alpha, beta = complex(2, -1), complex(1, 3)
    got = gemm(engine_ctx, opA, opB, A, B, alpha, beta, C0)
    ref = alpha * (opm(A, opA) @ opm(B, opB)) + beta * C0
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("opA,opB", [("N", "N"), ("N", "C"), ("C", "N"), ("T", "T")])
def test_random_products(engine_ctx, opA, opB):
    rng = np.random.default_rng(3)
    M, N, K = 520, 260, 777
    Am = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
    Bm = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
    A = Am if opA == "N" else (Am.T if opA == "T" else Am.conj().T)
    B = Bm if opB == "N" else (Bm.T if opB == "T" else Bm.conj().T)
    got = gemm(engine_ctx, opA, opB, A, B, complex(1, 0), complex(0, 0), np.zeros((M, N), complex))
    ref = Am @ Bm
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-13
