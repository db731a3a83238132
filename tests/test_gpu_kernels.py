"""FP64 kernel parity: the CUDA Heff / push / factorization kernels against the oracle.

Tolerance: 1e-12 relative (FP64 contractions, summation order differs)."""
import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rand_c(rng, *shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


MODELS = {
    "tfim": O.tfim_hamiltonian,
    "xxz": O.heisenberg_hamiltonian,
    "hubbard": O.hubbard_hamiltonian,
}


@pytest.mark.parametrize("model,D,N", [("tfim", 16, 1), ("tfim", 1, 1), ("xxz", 33, 2), ("xxz", 5, 1),
                                       ("hubbard", 20, 2), ("hubbard", 3, 1), ("tfim", 70, 1)])
def test_ac_c_apply_random_envs(ctx, model, D, N):
    oH = MODELS[model]()
    oH = O.SchurMPO([oH.Ws[0]] * N)
    w = oH.Ws[0].shape[0]
    d = oH.Ws[0].shape[1]
    rng = np.random.default_rng(D * 7 + N)
    opsi = O.CanonicalIMPS([rand_c(rng, D, d, D) for _ in range(N)], [rand_c(rng, D, d, D) for _ in range(N)],
                           [rand_c(rng, D, D) for _ in range(N)], [rand_c(rng, D, d, D) for _ in range(N)])
    oenvs = O.DMRGCache([rand_c(rng, D, w, D) for _ in range(N)], [rand_c(rng, D, w, D) for _ in range(N)])
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = upload_envs(psi, H, oenvs)
    for site in range(1, N + 1):
        x = rand_c(rng, D, d, D)
        y = imps.AC_hamiltonian(site, psi, H, psi, envs)(x)
        yref = O.ac_apply(oenvs.lefts[site - 1], oH[site - 1], oenvs.rights[site - 1], x)
        assert rel(y, yref) < TOL
        c = rand_c(rng, D, D)
        yc = imps.C_hamiltonian(site, psi, H, psi, envs)(c)
        ycref = O.c_apply(oenvs.lefts[site % N], oenvs.rights[site - 1], c)
        assert rel(yc, ycref) < TOL


@pytest.mark.parametrize("Dl,d,Dr", [(7, 2, 9), (16, 2, 16), (1, 3, 2), (40, 4, 37)])
def test_identity_pushes(ctx, Dl, d, Dr):
    rng = np.random.default_rng(Dl + 10 * Dr)
    A = rand_c(rng, Dl, d, Dr)
    B = rand_c(rng, Dl, d, Dr)
    Lm = rand_c(rng, Dl, Dl)
    Rm = rand_c(rng, Dr, Dr)
    assert rel(imps.push_env_left(Lm, A, B), O.push_env_left(Lm, A, B)) < TOL
    assert rel(imps.push_env_right(Rm, A, B), O.push_env_right(Rm, A, B)) < TOL


@pytest.mark.parametrize("model,Dl,Dr", [("tfim", 9, 11), ("xxz", 16, 16), ("hubbard", 13, 10)])
def test_mpo_pushes(ctx, model, Dl, Dr):
    oH = MODELS[model]()
    W = oH.Ws[0]
    w, d = W.shape[0], W.shape[1]
    rng = np.random.default_rng(Dl * Dr)
    A = rand_c(rng, Dl, d, Dr)
    Lm = rand_c(rng, Dl, w, Dl)
    Rm = rand_c(rng, Dr, w, Dr)
    H = to_device_mpo(oH)
    assert rel(imps.push_mpo_left(Lm, H, 1, A), O.push_mpo_left(Lm, W, A)) < TOL
    assert rel(imps.push_mpo_right(Rm, H, 1, A), O.push_mpo_right(Rm, W, A)) < TOL


@pytest.mark.parametrize("m,n", [(12, 5), (64, 64), (5, 12), (1, 1), (300, 129)])
def test_qrpos_lqpos(ctx, m, n):
    rng = np.random.default_rng(m * n)
    M = rand_c(rng, m, n)
    Q, R = imps.qrpos(M)
    Qr, Rr = O.qrpos(M)
    assert rel(Q @ R, M) < 1e-13
    assert rel(Q, Qr) < 1e-10 and rel(R, Rr) < 1e-10
    assert np.all(np.abs(np.diag(R).imag) < 1e-12) and np.all(np.diag(R).real >= 0)
    Lf, Qq = imps.lqpos(M)
    Lr, Qqr = O.lqpos(M)
    assert rel(Lf @ Qq, M) < 1e-13
    assert rel(Lf, Lr) < 1e-10 and rel(Qq, Qqr) < 1e-10


def test_regauge(ctx):
    rng = np.random.default_rng(5)
    AC = rand_c(rng, 10, 2, 12)
    Cm = rand_c(rng, 12, 12)
    assert rel(imps.regauge(AC, Cm), O.regauge(AC, Cm)) < 1e-10


def test_shape_errors(ctx):
    H = imps.tfim_hamiltonian()
    psi = imps.CanonicalIMPS(ctx, [2], [4])
    envs = imps.DMRGCache(psi, H, build=False)
    with pytest.raises(imps.DimensionMismatch):
        imps.AC_hamiltonian(1, psi, H, psi, envs)(np.zeros((4, 2, 5), complex))
    with pytest.raises(imps.DimensionMismatch):
        imps.DMRGCache(psi, imps.hubbard_hamiltonian(), build=False)
