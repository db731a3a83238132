"""Oracle MPO application mult(W, psi, VOMPS) (src/algorithms/arithmetics/mult.jl,
arithmetics/envs.jl:51-93) on the CPU: the identity MPO returns the state, and one
W^II step agrees with a TDVP step to second order in the time step."""
import numpy as np
import pytest

import oracle as O


@pytest.fixture(scope="module")
def tfim_gs():
    H0 = O.tfim_hamiltonian(J=1.0, h=0.5)
    psi, _, _ = O.find_groundstate(O.randomimps([2], D=8, seed=4), H0, O.VUMPS(D=8, maxiter=200, tol=1e-10))
    return psi


def test_identity_mpo_returns_the_state(tfim_gs):
    I = [np.asfortranarray(np.eye(2, dtype=complex).reshape(1, 2, 1, 2))]
    y, envs, info = O.mult(I, tfim_gs, O.VOMPS(D=8, maxiter=20, tol=1e-10))
    assert info["converged"]
    assert abs(abs(O.state_dot(tfim_gs, y)) - 1) < 1e-10
    assert O.mult_galerkin(envs, y) == info["itererr"]


def test_wii_step_matches_tdvp_step(tfim_gs):
    H1 = O.tfim_hamiltonian(J=1.0, h=1.5)
    W = O.timeevompo(H1, -1j * 0.01, "WII")
    y, envs, info = O.mult(W, tfim_gs, O.VOMPS(D=8, maxiter=50, tol=1e-10))
    assert info["converged"] and info["losses"][-1] <= 1e-10
    p1, _ = O.timestep(tfim_gs, H1, -0.01j, O.TDVP(), O.build_envs(tfim_gs, H1))
    sx = O.sigma("x")
    moved = abs(O.local_expectation1(tfim_gs, 0, sx) - O.local_expectation1(p1, 0, sx))
    assert moved > 1e-4
    assert abs(O.local_expectation1(y, 0, sx) - O.local_expectation1(p1, 0, sx)) < 1e-6


def test_two_site_cell_and_ternary_push_identities():
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi, _, _ = O.find_groundstate(O.randomimps([2, 2], D=6, seed=21), H, O.VUMPS(D=6, maxiter=200, tol=1e-9))
    W = O.timeevompo(H, -1j * 0.02, "WII")
    y, envs, info = O.mult(W, psi, O.VOMPS(D=6, maxiter=50, tol=1e-9))
    assert info["converged"]
    p1, _ = O.timestep(psi, H, -0.02j, O.TDVP(), O.build_envs(psi, H))
    assert abs(O.state_dot(y, p1)) > 1 - 1e-8
    # the ternary pushes reduce to the MPO pushes when bra = ket
    rng = np.random.default_rng(3)
    L = rng.standard_normal((6, 4, 6)) + 1j * rng.standard_normal((6, 4, 6))
    A = psi.AL[0]
    np.testing.assert_allclose(O.push_ternary_left(L, A, W[0], A), O.push_mpo_left(L, W[0], A), atol=1e-12)
    np.testing.assert_allclose(O.push_ternary_right(L, A, W[0], A), O.push_mpo_right(L, W[0], A), atol=1e-12)


def test_reference_identity_mpo_on_random_state():
    # test/algorithms/api.jl:502-508: the identity MPO applied to a random N=1 D=6 state at
    # D = 6 returns it (|<y|psi>| = 1 within 1e-6)
    psi0 = O.randomimps([2], D=6, seed=42)
    I = [np.asfortranarray(np.eye(2, dtype=complex).reshape(1, 2, 1, 2))]
    y, _, _ = O.mult(I, psi0, O.VOMPS(D=6, maxiter=50, tol=1e-10))
    assert abs(abs(O.state_dot(y, psi0)) - 1) < 1e-6


def test_reference_lossless_bond_equals_naive_product():
    # test/algorithms/arithmetics.jl:290-297: at the lossless bond dimension the result is
    # the naive product W . psi (fidelity > 1 - 1e-8)
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    W = O.timeevompo(H, -0.05j, "WII")
    psi = O.randomimps([2, 2], D=3, seed=9)
    As = []
    for l in range(2):
        wl, u, wr, _ = W[l].shape
        bl, _, br = psi.AL[l].shape
        B5 = np.einsum("wurd,bdc->wburc", W[l], psi.AL[l])
        As.append(np.asfortranarray(B5.reshape((wl * bl, u, wr * br), order="F")))
    ref = O.canonical_from_sites(As)
    y, _, info = O.mult(W, psi, O.VOMPS(D=12, maxiter=300, tol=1e-10))
    assert max(a.shape[2] for a in y.AL) == 12
    assert abs(O.state_dot(y, ref)) > 1 - 1e-8
