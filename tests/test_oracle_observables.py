"""The oracle's dense-MPO channel, correlators and entanglement observables (CPU),
against the reference's own tests: test/algorithms/observables.jl:1-40 (product-state
correlators, Heisenberg nearest-neighbour sign, entropy bounds, normalised spectra),
test/algorithms/api.jl:512-535 (correlator head value equals the two-site local
expectation; product-state entropies vanish) and the identity-MPO normalisation of
the dense channel (the local contraction of every site is 1, so <I> = N)."""
import numpy as np
import pytest

import oracle as O


def prod_state(dims, idx):
    ALs = []
    for d, k in zip(dims, idx):
        A = O.fzeros((1, d, 1))
        A[0, k, 0] = 1.0
        ALs.append(A)
    return O.canonical_from_AL(ALs, np.eye(1, dtype=complex))


def test_product_state_correlators_and_entropy():
    Z, X = O.sigma("z"), O.sigma("x")
    up = prod_state([2, 2], [0, 0])
    C = O.correlator(up, Z, Z, 1, range(2, 6))
    assert np.all(np.abs(C - 1) < 1e-12)
    Cx = O.correlator(up, X, X, 1, range(2, 5))
    assert np.all(np.abs(Cx) < 1e-12)
    neel = prod_state([2, 2], [0, 1])
    for loc in (1, 2):
        assert abs(O.entropy(neel, loc)) < 1e-12
        assert abs(O.entanglement_spectrum(neel, loc).sum() - 1) < 1e-12


@pytest.fixture(scope="module")
def heis():
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi, envs, _ = O.find_groundstate(O.randomimps([2, 2], D=12, seed=1), H,
                                      O.VUMPS(D=12, maxiter=200, tol=1e-9))
    return psi, envs, H


def test_heisenberg_correlator_head_and_entropy(heis):
    psi, envs, H = heis
    Sz = O.spin("z")
    G = O.correlator(psi, Sz, Sz, 1, range(2, 7))
    assert G[0].real < 0
    assert np.all(G.real < 0.26)
    # head value == the two-site local expectation <Sz_1 Sz_2> (api.jl:521-522)
    A2 = np.einsum("asm,mtb->astb", psi.AC[0], psi.AR[1])
    e12 = np.einsum("astb,su,tv,auvb->", A2.conj(), Sz, Sz, A2) / O.state_dot(psi, psi)
    assert abs(G[0] - e12) < 1e-10
    S = O.entropy(psi)
    assert 0.5 < S < 2.0
    p = O.entanglement_spectrum(psi)
    assert abs(p.sum() - 1) < 1e-10 and p[0] >= p[-1]
    assert O.entropy(psi, alpha=2.0) <= S + 1e-12


def test_dense_channel_identity_mpo(heis):
    psi = heis[0]
    Id = [np.asfortranarray(np.eye(2, dtype=complex).reshape(1, 2, 1, 2)) for _ in range(2)]
    envs = O.build_envs_dense(psi, Id)
    assert abs(O.expectationvalue_dense(psi, Id, envs) - 2.0) < 1e-10
    lam, L = O.dominant_env(psi)
    assert abs(lam - 1) < 1e-10 and abs(np.linalg.norm(L) - 1) < 1e-12
