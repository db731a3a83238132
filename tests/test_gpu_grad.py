"""Energy gradients on the GPU: the CUDA adjoint contractions against the oracle,
against central finite differences of the GPU energy, and against the
Hellmann-Feynman value at a converged ground state."""
import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu


def test_gradients_match_oracle(ctx):
    oH = O.SchurMPO([O.hubbard_hamiltonian().Ws[0]] * 2)
    opsi = O.randomimps([4, 4], D=12, seed=9)
    oenvs = O.build_envs(opsi, oH, tol=1e-12)
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = upload_envs(psi, H, oenvs)
    G = imps.energy_gradient_mpo(psi, H, envs)
    Go = O.energy_grad_mpo(opsi, oH, oenvs)
    g = imps.energy_gradient_AL(psi, H, envs)
    go = O.energy_grad_al(opsi, oH, oenvs)
    for l in range(2):
        assert rel(G[l], Go[l]) < 1e-11
        assert rel(g[l], go[l]) < 1e-11


def tfim(J, h):
    return imps.tfim_hamiltonian(J, h)


def test_coupling_gradient_hellmann_feynman_and_fd(ctx):
    J, h, dl, D = 1.0, 0.6, 1e-5, 16
    alg = imps.VUMPS(D=D, maxiter=400, tol=1e-12)
    psi, envs, info = imps.find_groundstate(imps.randomimps([2], D=D, seed=4, ctx=ctx), tfim(J, h), alg)
    dW = [(tfim(J, h + dl).Ws[0] - tfim(J, h - dl).Ws[0]) / (2 * dl)]
    dEdh = imps.coupling_gradient(psi, tfim(J, h), dW, envs).real
    hf = -imps.expectationvalue(psi, (1, O.sigma("z"))).real
    assert abs(dEdh - hf) < 1e-9
    ep = imps.find_groundstate(psi, tfim(J, h + dl), alg)
    em = imps.find_groundstate(psi, tfim(J, h - dl), alg)
    fd = (imps.expectationvalue(ep[0], tfim(J, h + dl), ep[1]).real
          - imps.expectationvalue(em[0], tfim(J, h - dl), em[1]).real) / (2 * dl)
    assert abs(fd - dEdh) < 1e-6


def test_al_gradient_directional_fd(ctx):
    H = imps.SparseIMPO([O.tfim_hamiltonian(1.0, 0.7).Ws[0]] * 2)
    psi = imps.randomimps([2, 2], D=6, seed=11, ctx=ctx)
    envs = imps.DMRGCache(psi, H, tol=1e-13)
    g = imps.energy_gradient_AL(psi, H, envs)
    rng = np.random.default_rng(5)
    AL = [psi.AL[l] for l in (1, 2)]
    X = [rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape) for a in AL]
    analytic = sum(2.0 * np.real(np.vdot(g[l], X[l])) for l in range(2))

    def e_of(As):
        p = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
        return imps.expectationvalue(p, H, imps.DMRGCache(p, H, tol=1e-13)).real
    eps = 1e-5
    fd = (e_of([AL[l] + eps * X[l] for l in range(2)]) - e_of([AL[l] - eps * X[l] for l in range(2)])) / (2 * eps)
    assert abs(fd - analytic) < 1e-6 * max(1.0, abs(analytic))
