"""Dense-MPO channel environments, correlators and entanglement spectra on the CUDA
path against the oracle (tests/test_oracle_observables.py pins the oracle on the
reference's own tests): the identity and dense-MPO dominant environments, the
DMRGCache(psi, ::DenseIMPO) build with its normalisation (identity MPO: <I> = N),
the dense expectation value of a random MPO, correlators of a Heisenberg ground state
and of product states (test/algorithms/observables.jl:1-40), and the entanglement
spectrum / entropies by the device Jacobi SVD against LAPACK singular values."""
import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
import oracle as O
from gpu_helpers import rel, upload_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def heis():
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi, _, _ = O.find_groundstate(O.randomimps([2, 2], D=12, seed=1), H, O.VUMPS(D=12, maxiter=200, tol=1e-9))
    return psi


def _phase(a, b):
    ov = np.vdot(b.ravel(), a.ravel())
    return a * (np.conj(ov) / abs(ov))


def test_dominant_env_identity_and_dense(ctx, heis):
    psi = upload_state(ctx, heis)
    for side in ("left", "right"):
        lam, L = imps.dominant_env(psi, side=side)
        lo, Lo = O.dominant_env(heis, None, side)
        assert abs(lam - lo) < 1e-10
        assert rel(_phase(L, Lo), Lo) < 1e-8
    rng = np.random.default_rng(4)
    Wd = [np.asfortranarray(rng.standard_normal((3, 2, 3, 2)) + 1j * rng.standard_normal((3, 2, 3, 2)))
          for _ in range(2)]
    W = imps.DenseIMPO(Wd)
    for side in ("left", "right"):
        lam, L = imps.dominant_env(psi, W, side=side)
        lo, Lo = O.dominant_env(heis, Wd, side)
        assert abs(lam - lo) < 1e-9 * abs(lo)
        assert rel(_phase(L, Lo), Lo) < 1e-7


def test_dense_envs_and_expectation(ctx, heis):
    psi = upload_state(ctx, heis)
    Id = imps.identityimpo([2, 2])
    assert abs(imps.expectationvalue(psi, Id) - 2.0) < 1e-10
    rng = np.random.default_rng(5)
    Wd = []
    for _ in range(2):
        X = rng.standard_normal((2, 2, 2, 2)) + 1j * rng.standard_normal((2, 2, 2, 2))
        Wd.append(np.asfortranarray(X + np.eye(2).reshape(1, 2, 1, 2)))
    W = imps.DenseIMPO(Wd)
    envs = imps.DMRGCache(psi, W)
    oenvs = O.build_envs_dense(heis, Wd)
    e = imps.expectationvalue(psi, W, envs)
    eo = O.expectationvalue_dense(heis, Wd, oenvs)
    assert abs(e - eo) < 1e-9 * max(1.0, abs(eo))


def test_correlators(ctx, heis):
    psi = upload_state(ctx, heis)
    Sz = O.spin("z")
    G = imps.correlator(psi, Sz, Sz, 1, range(2, 7))
    Go = O.correlator(heis, Sz, Sz, 1, range(2, 7))
    assert np.max(np.abs(G - Go)) < 1e-11
    assert G[0].real < 0
    # single j
    assert abs(imps.correlator(psi, Sz, Sz, 1, 3) - O.correlator(heis, Sz, Sz, 1, [3])[0]) < 1e-11
    with pytest.raises(imps.ArgumentError):
        imps.correlator(psi, Sz, Sz, 2, range(2, 4))


def test_product_state_correlators_and_entropy(ctx):
    Z = O.sigma("z")
    ALs = []
    for k in (0, 0):
        A = np.zeros((1, 2, 1), dtype=complex, order="F")
        A[0, k, 0] = 1.0
        ALs.append(A)
    psi = imps.CanonicalIMPS.from_AL(ALs, np.eye(1, dtype=complex), ctx=ctx)
    C = imps.correlator(psi, Z, Z, 1, range(2, 6))
    assert np.all(np.abs(C - 1) < 1e-12)
    assert abs(imps.entropy(psi, 1)) < 1e-12
    assert abs(imps.entanglement_spectrum(psi, 2).sum() - 1) < 1e-12


@pytest.mark.parametrize("D,seed", [(12, 1), (37, 2), (128, 3)])
def test_entanglement_spectrum_against_lapack(ctx, D, seed):
    opsi = O.randomimps([2, 2], D=D, seed=seed)
    psi = upload_state(ctx, opsi)
    for loc in (1, 2):
        p = imps.entanglement_spectrum(psi, loc)
        po = O.entanglement_spectrum(opsi, loc)
        assert np.max(np.abs(p - po)) < 1e-13
        assert abs(imps.entropy(psi, loc) - O.entropy(opsi, loc)) < 1e-11
        assert abs(imps.entropy(psi, loc, alpha=2.0) - O.entropy(opsi, loc, alpha=2.0)) < 1e-11


@pytest.mark.parametrize("m,n,kmax", [(20, 7, 0), (7, 20, 0), (64, 64, 10), (300, 120, 0), (33, 1, 0)])
def test_tsvd_against_lapack(ctx, m, n, kmax):
    rng = np.random.default_rng(m + n)
    M = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    U, s, V = imps.tsvd(M, kmax, ctx=ctx)
    so = np.linalg.svd(M, compute_uv=False)
    k = len(s)
    assert k == (kmax if kmax else min(m, n))
    assert np.allclose(s, so[:k], rtol=1e-12, atol=1e-12 * so[0])
    assert np.linalg.norm(U.conj().T @ U - np.eye(k)) < 1e-12 * k
    assert np.linalg.norm(V.conj().T @ V - np.eye(k)) < 1e-12 * k
    if kmax == 0:
        assert np.linalg.norm((U * s) @ V.conj().T - M) < 1e-12 * np.linalg.norm(M)
    else:
        # best rank-k approximation error = the discarded singular values
        err = np.linalg.norm((U * s) @ V.conj().T - M)
        assert abs(err - np.linalg.norm(so[k:])) < 1e-10 * np.linalg.norm(M)
