"""The Krylov solvers' small FP64 eigenproblems (csrc/smallla.cu) on the host.

smallla.cu is plain host C++ (the projected Ritz / Schur problems of the Lanczos,
Arnoldi and exponentiate solvers run on the CPU thread that drives the stream), so
it is compiled here with g++ into a throwaway library and checked against LAPACK
(numpy): Hermitian eigenpairs including the thick-restart arrowhead shape,
degenerate spectra, and the sorted complex Schur form used by the Krylov-Schur
restart of the Arnoldi solver.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    out = tmp_path_factory.mktemp("smallla") / "libsmallla.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-x", "c++", "-I", "/usr/local/cuda/include",
                    os.path.join(HERE, "smallla_harness.cpp"), "-o", str(out)], check=True)
    lb = C.CDLL(str(out))
    DP = C.POINTER(C.c_double)
    for f in ("h_herm_eig", "h_schur_sorted", "h_gen_eig"):
        getattr(lb, f).argtypes = [C.c_int, DP, DP, DP]
    return lb


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _herm(lib, A):
    n = A.shape[0]
    A = np.asfortranarray(A, dtype=complex)
    w = np.zeros(n)
    V = np.zeros((n, n), dtype=complex, order="F")
    lib.h_herm_eig(n, _p(A), _p(w), _p(V))
    return w, V


def _rand(rng, n):
    return rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))


@pytest.mark.parametrize("n", [1, 2, 3, 7, 30, 64])
def test_herm_eig_matches_lapack(lib, n):
    rng = np.random.default_rng(n)
    X = _rand(rng, n)
    A = X + X.conj().T
    w, V = _herm(lib, A)
    assert np.allclose(w, np.linalg.eigvalsh(A), atol=1e-12 * max(1.0, np.abs(w).max()))
    assert np.all(np.diff(w) >= 0)
    assert np.linalg.norm(V.conj().T @ V - np.eye(n)) < 1e-12 * n
    assert np.linalg.norm(A @ V - V * w) < 1e-12 * n * np.linalg.norm(A)


def test_herm_eig_lanczos_shapes(lib):
    rng = np.random.default_rng(7)
    # tridiagonal with complex couplings, and the arrowhead of a thick restart
    n, keep = 30, 18
    T = np.diag(rng.standard_normal(n)).astype(complex)
    off = rng.standard_normal(n - 1) * np.exp(1j * rng.uniform(0, 2 * np.pi, n - 1))
    T += np.diag(off, -1) + np.diag(off.conj(), 1)
    Ar = np.zeros((n, n), dtype=complex)
    Ar[:keep, :keep] = np.diag(np.sort(rng.standard_normal(keep)))
    Ar[keep, :keep] = rng.standard_normal(keep) + 1j * rng.standard_normal(keep)
    Ar[:keep, keep] = Ar[keep, :keep].conj()
    Ar[keep:, keep:] = T[keep:, keep:]
    for A in (T, Ar):
        w, V = _herm(lib, A)
        assert np.allclose(w, np.linalg.eigvalsh(A), atol=1e-12)
        assert np.linalg.norm(A @ V - V * w) < 1e-11


def test_herm_eig_degenerate_and_diagonal(lib):
    A = np.diag([2.0, -1.0, 2.0, 0.0, -1.0]).astype(complex)
    w, V = _herm(lib, A)
    assert np.allclose(w, [-1, -1, 0, 2, 2])
    assert np.linalg.norm(A @ V - V * w) < 1e-14
    w, V = _herm(lib, np.zeros((4, 4), dtype=complex))
    assert np.allclose(w, 0) and np.allclose(V.conj().T @ V, np.eye(4))


@pytest.mark.parametrize("n", [1, 2, 5, 30])
def test_schur_sorted(lib, n):
    rng = np.random.default_rng(100 + n)
    H = np.asfortranarray(np.triu(_rand(rng, n), -1))  # Hessenberg, as Arnoldi makes it
    for M in (H, np.asfortranarray(_rand(rng, n))):
        T = np.zeros((n, n), dtype=complex, order="F")
        Z = np.zeros((n, n), dtype=complex, order="F")
        lib.h_schur_sorted(n, _p(M), _p(T), _p(Z))
        assert np.allclose(np.tril(T, -1), 0)
        assert np.linalg.norm(Z.conj().T @ Z - np.eye(n)) < 1e-12 * n
        assert np.linalg.norm(Z @ T @ Z.conj().T - M) < 1e-12 * n * np.linalg.norm(M)
        d = np.abs(np.diag(T))
        assert np.all(np.diff(d) <= 1e-12 * d.max())
        lam = np.linalg.eigvals(M)
        assert np.allclose(np.sort(np.abs(lam))[::-1], d, atol=1e-10 * d.max())
        # the leading k Schur vectors span an invariant subspace
        k = max(1, n // 2)
        R = M @ Z[:, :k] - Z[:, :k] @ T[:k, :k]
        assert np.linalg.norm(R) < 1e-11 * n * np.linalg.norm(M)


def test_gen_eig(lib):
    rng = np.random.default_rng(3)
    n = 20
    M = np.asfortranarray(_rand(rng, n))
    lam = np.zeros(n, dtype=complex)
    Y = np.zeros((n, n), dtype=complex, order="F")
    lib.h_gen_eig(n, _p(M), _p(lam), _p(Y))
    assert np.linalg.norm(M @ Y - Y * lam) < 1e-10 * np.linalg.norm(M)
    assert np.allclose(np.sort_complex(lam), np.sort_complex(np.linalg.eigvals(M)), atol=1e-10)
