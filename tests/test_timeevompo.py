"""W^I / W^II time-evolution MPOs (timeevompo, src/algorithms/timeevo/w1w2.jl:26-45).

The reference's per-site kernel lives in an unvendored package, so the oracle
restates the published construction (arXiv:1407.1832); tensor-level parity is
unpinned, and the reference's own tests pin it only through energy conservation under
the exact application (test/operators/w1w2.jl:1-33, test/algorithms/tdvp.jl:36-43, at
their tolerances 1e-10 / 1e-4 / 1e-6).  The oracle is further checked by the physics, the periodic-trace ring operator of the MPO matching
exp(delta H) of the ring up to O(delta^2) (error ratio 4 when delta halves) and the
identity Hamiltonian giving the identity MPO (test/operators/w1w2.jl:11-17), and the
library's host routine behind imps_timeevompo_tensor is checked against the oracle
(no device needed)."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as O
import oracle.imps_oracle as OI


def ring_hamiltonian(W, L):
    D, C, B, A = OI._schur_blocks(W)
    d = W.shape[1]

    def op(ops):
        M = np.array([[1.0 + 0j]])
        for x in range(L):
            M = np.kron(M, ops.get(x, np.eye(d)))
        return M
    H = sum(op({x: D}) for x in range(L))
    for x in range(L):
        for b in range(len(C)):
            H = H + op({x: C[b], (x + 1) % L: B[b]})
    return H


@pytest.mark.parametrize("model", ["tfim", "xxz"])
@pytest.mark.parametrize("alg", ["WI", "WII"])
def test_ring_propagator_error_is_second_order(model, alg):
    H = {"tfim": O.tfim_hamiltonian, "xxz": O.heisenberg_hamiltonian}[model]()
    L = 4
    Hr = ring_hamiltonian(H.Ws[0], L)
    errs = []
    for dt in (0.04, 0.02, 0.01):
        for delta in (-1j * dt,):
            U = O.mpo_ring(O.timeevompo(H, delta, alg), L)
            errs.append(np.linalg.norm(U - sl.expm(delta * Hr)) / np.linalg.norm(U))
    assert errs[-1] < 1e-3
    assert 3.8 < errs[0] / errs[1] < 4.2 and 3.8 < errs[1] / errs[2] < 4.2


def test_identity_hamiltonian_gives_identity():
    W = O.mpohamiltonian(np.zeros((2, 2), complex), [])
    for alg in ("WI", "WII"):
        U = O.timeevompo(O.SchurMPO([W]), -0.01j, alg)[0]
        assert U.shape == (1, 2, 1, 2)
        assert np.allclose(U[0, :, 0, :], np.eye(2), atol=1e-15)


@pytest.mark.parametrize("alg", ["WI", "WII"])
def test_library_tensor_matches_oracle(alg):
    import infinitempsalgorithms_b200 as imps
    for H, oH in ((imps.tfim_hamiltonian(0.7, 1.3), O.tfim_hamiltonian(0.7, 1.3)),
                  (imps.hubbard_hamiltonian(), O.hubbard_hamiltonian()),
                  (imps.heisenberg_hamiltonian(), O.heisenberg_hamiltonian())):
        for delta in (-0.05j, -0.03, 0.02 - 0.04j):
            got = imps.timeevompo(H, delta, alg).Ws[0]
            ref = O.timeevompo(oH, delta, alg)[0]
            assert np.max(np.abs(got - ref)) < 1e-13


def _apply_exact(Ws, psi):
    """``CanonicalIMPS((W * DenseIMPS(psi.AL)).As)`` (test/operators/w1w2.jl:11): the
    uncompressed product, site tensors ``B[(wl, bl), u, (wr, br)] = sum_d W[wl,u,wr,d]
    AL[bl,d,br]`` (``operators/linalg.jl:15-20``), then canonical form."""
    As = []
    for l, A in enumerate(psi.AL):
        W = Ws[l % len(Ws)]
        wl, u, wr, _ = W.shape
        bl, _, br = A.shape
        B5 = np.einsum("wurd,bdc->wburc", W, A)
        As.append(np.asfortranarray(B5.reshape((wl * bl, u, wr * br), order="F")))
    return O.canonical_from_sites(As)


def test_reference_energy_conservation_random_state():
    # test/operators/w1w2.jl:1-33: a random D=8 two-site state, dt = 0.01; the identity
    # Hamiltonian's W^I leaves the energy unchanged (1e-10), W^II and W^I keep it within 1e-4
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi0 = O.randomimps([2, 2], D=8, seed=61)
    e0 = O.expectationvalue(psi0, H, O.build_envs(psi0, H)).real / 2
    empty = O.SchurMPO([O.mpohamiltonian(np.zeros((2, 2), complex), [])] * 2)
    out = _apply_exact(O.timeevompo(empty, -0.01j, "WI"), psi0)
    assert abs(O.expectationvalue(out, H, O.build_envs(out, H)).real / 2 - e0) < 1e-10
    for alg in ("WII", "WI"):
        out = _apply_exact(O.timeevompo(H, -0.01j, alg), psi0)
        assert abs(O.expectationvalue(out, H, O.build_envs(out, H)).real / 2 - e0) < 1e-4


def test_reference_energy_conservation_ground_state():
    # test/algorithms/tdvp.jl:36-43: from the VUMPS ground state, W^II at dt = 0.01 keeps
    # the energy within 1e-6
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi, envs, _ = O.find_groundstate(O.randomimps([2, 2], D=8, seed=62), H, O.VUMPS(D=8, maxiter=200, tol=1e-10))
    e0 = O.expectationvalue(psi, H, envs).real / 2
    out = _apply_exact(O.timeevompo(H, -0.01j, "WII"), psi)
    assert abs(O.expectationvalue(out, H, O.build_envs(out, H)).real / 2 - e0) < 1e-6
