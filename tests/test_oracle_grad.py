"""The oracle's energy gradients against central finite differences (CPU only).

The reference has no gradient code, so these pin the oracle by finite
differences of its own energy functional and by the Hellmann-Feynman theorem at
a converged ground state; the GPU tests then compare the CUDA gradients with it."""
import numpy as np
import pytest

import oracle as O


def tfim_cell(J, h, N):
    return O.SchurMPO([O.tfim_hamiltonian(J, h).Ws[0]] * N)


def energy_fixed_state(psi, H):
    envs = O.build_envs(psi, H, tol=1e-13)
    return O.expectationvalue(psi, H, envs)


@pytest.mark.parametrize("N", [1, 2])
def test_mpo_gradient_matches_central_differences(N):
    psi = O.randomimps([2] * N, D=6, seed=3)
    J, h, dl = 1.0, 0.7, 1e-5
    H = tfim_cell(J, h, N)
    envs = O.build_envs(psi, H, tol=1e-13)
    G = O.energy_grad_mpo(psi, H, envs)
    for which in ("h", "J"):
        f = (lambda t: tfim_cell(J, t, N)) if which == "h" else (lambda t: tfim_cell(t, h, N))
        t0 = h if which == "h" else J
        Hp, Hm = f(t0 + dl), f(t0 - dl)
        dW = [(Hp.Ws[l] - Hm.Ws[l]) / (2 * dl) for l in range(N)]
        analytic = sum(np.sum(dW[l] * G[l]) for l in range(N))
        fd = (energy_fixed_state(psi, Hp) - energy_fixed_state(psi, Hm)) / (2 * dl)
        assert abs(analytic - fd) < 1e-8 * max(1.0, abs(fd))


@pytest.mark.parametrize("N", [1, 2])
def test_al_gradient_matches_central_differences(N):
    H = tfim_cell(1.0, 0.7, N)
    psi = O.randomimps([2] * N, D=5, seed=11)
    envs = O.build_envs(psi, H, tol=1e-13)
    g = O.energy_grad_al(psi, H, envs)
    rng = np.random.default_rng(5)
    X = [np.asfortranarray(rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)) for a in psi.AL]
    analytic = sum(2.0 * np.real(np.vdot(g[l], X[l])) for l in range(N))

    def e_of(As):
        p = O.canonical_from_sites(As)
        return energy_fixed_state(p, H).real
    errs = []
    for eps in (1e-4, 1e-5):
        fd = (e_of([psi.AL[l] + eps * X[l] for l in range(N)]) - e_of([psi.AL[l] - eps * X[l] for l in range(N)])) / (2 * eps)
        errs.append(abs(fd - analytic))
    # central differences converge as eps^2 onto the analytic value
    assert errs[1] < 1e-6 * abs(analytic) and errs[1] < 0.05 * errs[0]


def test_hellmann_feynman_at_ground_state():
    # at a VUMPS fixed point dE0/dh = <dH/dh> = -<sigma_z> per site (H = -J xx - h z)
    J, h, dl, D = 1.0, 0.6, 1e-5, 8
    H = tfim_cell(J, h, 1)
    alg = O.VUMPS(D=D, maxiter=400, tol=1e-12)
    psi, envs, info = O.find_groundstate(O.randomimps([2], D=D, seed=4), H, alg)
    G = O.energy_grad_mpo(psi, H, envs)
    dW = (tfim_cell(J, h + dl, 1).Ws[0] - tfim_cell(J, h - dl, 1).Ws[0]) / (2 * dl)
    dEdh = np.sum(dW * G[0]).real
    hf = -O.local_expectation1(psi, 0, O.sigma("z")).real
    assert abs(dEdh - hf) < 1e-10
    psi_p, envs_p, _ = O.find_groundstate(psi, tfim_cell(J, h + dl, 1), alg)
    psi_m, envs_m, _ = O.find_groundstate(psi, tfim_cell(J, h - dl, 1), alg)
    fd = (O.expectationvalue(psi_p, tfim_cell(J, h + dl, 1), envs_p).real
          - O.expectationvalue(psi_m, tfim_cell(J, h - dl, 1), envs_m).real) / (2 * dl)
    assert abs(fd - dEdh) < 1e-6
