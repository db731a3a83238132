"""Non-uniform bond and physical dimensions in the oracle (CPU only), after the
reference's test/algorithms/envs.jl:30-126: environments and energies on a unit
cell with bond profile [2, 4, 2], invariance of the energy under zero-padding
of one bond (same physical state, extra Schmidt directions of weight zero), and
a unit cell with physical dimensions [2, 3, 2]."""
import numpy as np

import oracle as O


def tfim_cell(J, h, N):
    return O.SchurMPO([O.tfim_hamiltonian(J, h).Ws[0]] * N)


def zext(A, n, axis):
    shape = list(A.shape)
    shape[axis] = n
    return np.asfortranarray(np.concatenate([A, np.zeros(shape, dtype=A.dtype)], axis=axis))


def complete_cols(Q, n, rng):
    # n new orthonormal columns orthogonal to the isometry Q
    Y = rng.standard_normal((Q.shape[0], n)) + 1j * rng.standard_normal((Q.shape[0], n))
    Y = Y - Q @ (Q.conj().T @ Y)
    q, _ = np.linalg.qr(Y)
    return np.asfortranarray(np.hstack([Q, q]))


def pad_bond(psi, b, n, rng):
    """Grow bond b (0-based, right of site b) by n zero-weight Schmidt directions."""
    N = len(psi)
    bn = (b + 1) % N
    AL, AR, Cs, AC = list(psi.AL), list(psi.AR), list(psi.C), list(psi.AC)
    chi = Cs[b].shape[0]
    dl, d, _ = AL[b].shape
    AL[b] = O.freshape(complete_cols(O.freshape(AL[b], (dl * d, chi)), n, rng), (dl, d, chi + n))
    AR[b] = zext(AR[b], n, 2)
    AL[bn] = zext(AL[bn], n, 0)
    _, d2, dr2 = AR[bn].shape
    R = O.freshape(AR[bn], (chi, d2 * dr2))
    Rt = complete_cols(np.asfortranarray(R.conj().T), n, rng)
    AR[bn] = O.freshape(np.asfortranarray(Rt.conj().T), (chi + n, d2, dr2))
    C = np.zeros((chi + n, chi + n), dtype=complex, order="F")
    C[:chi, :chi] = Cs[b]
    Cs[b] = C
    AC[b] = zext(AC[b], n, 2)
    AC[bn] = zext(AC[bn], n, 0)
    return O.CanonicalIMPS(AL, AR, Cs, AC)


def test_nonuniform_profile_envs_and_energy():
    rng = np.random.default_rng(7)
    chi = [2, 4, 2]
    N = 3
    ALs = []
    for l in range(N):
        dl, dr = chi[(l - 1) % N], chi[l]
        M = rng.standard_normal((dl * 2, dr)) + 1j * rng.standard_normal((dl * 2, dr))
        q, _ = np.linalg.qr(M)
        ALs.append(O.freshape(np.asfortranarray(q[:, :dr]), (dl, 2, dr)))
    psi = O.canonical_from_AL(ALs, np.eye(chi[N - 1], dtype=complex))
    H = tfim_cell(1.0, 1.3, N)
    envs = O.build_envs(psi, H)
    # the left environment of site l lives on bond l-1, the right one on bond l
    assert [envs.lefts[l].shape[0] for l in range(N)] == [2, 2, 4]
    assert [envs.rights[l].shape[0] for l in range(N)] == [2, 4, 2]
    assert np.isfinite(O.expectationvalue(psi, H, envs).real)


def test_zero_padding_leaves_energy_unchanged():
    # test/algorithms/envs.jl:61-66: pad bond 2 by one direction; |E_padded - E| < 1e-10
    rng = np.random.default_rng(3)
    H = tfim_cell(1.0, 1.3, 3)
    psi = O.randomimps([2, 2, 2], D=4, seed=13)
    E0 = O.expectationvalue(psi, H, O.build_envs(psi, H)).real
    psp = pad_bond(psi, 1, 1, rng)
    assert [psp.C[l].shape[0] for l in range(3)] == [4, 5, 4]
    # AL / AR stay isometric after padding
    for l in range(3):
        dl, d, dr = psp.AL[l].shape
        A = O.freshape(psp.AL[l], (dl * d, dr))
        assert np.allclose(A.conj().T @ A, np.eye(dr), atol=1e-12)
        B = O.freshape(psp.AR[l], (dl, d * dr))
        assert np.allclose(B @ B.conj().T, np.eye(dl), atol=1e-12)
    Ep = O.expectationvalue(psp, H, O.build_envs(psp, H)).real
    assert abs(Ep - E0) < 1e-10


def test_heterogeneous_physical_dims():
    # test/algorithms/envs.jl:75-126: unit cell with d = [2, 3, 2]
    dims = [2, 3, 2]
    psi = O.randomimps(dims, D=4, seed=3)
    assert abs(abs(O.state_dot(psi, psi)) - 1) < 1e-10
    for l, d in enumerate(dims):
        assert abs(O.local_expectation1(psi, l, np.eye(d)).real - 1) < 1e-10
    rng = np.random.default_rng(3)
    hd = []
    for d in dims:
        h = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        hd.append((h + h.conj().T) / 2)
    H = O.SchurMPO([O.mpohamiltonian(h, []) for h in hd])
    e0 = O.expectationvalue(psi, H, O.build_envs(psi, H)).real
    assert np.isfinite(e0)
    # adding lambda_l * I on every site shifts the energy per unit cell by sum(lambda)
    Hs = O.SchurMPO([O.mpohamiltonian(h + np.eye(h.shape[0]), []) for h in hd])
    e1 = O.expectationvalue(psi, Hs, O.build_envs(psi, Hs)).real
    assert abs(e1 - e0 - 3.0) < 1e-10


def test_heterogeneous_product_ground_state():
    # diagonal on-site fields: the ground state is a product state, E = sum of minima
    lams = [np.array([-2.0, 1.0]), np.array([-3.0, 0.0, 2.0]), np.array([-2.0, 1.0])]
    H = O.SchurMPO([O.mpohamiltonian(np.diag(l).astype(complex), []) for l in lams])
    ALs = []
    for l in lams:
        A = O.fzeros((1, len(l), 1))
        A[0, int(np.argmin(l)), 0] = 1.0
        ALs.append(A)
    psi0 = O.canonical_from_AL(ALs, np.eye(1, dtype=complex))
    psi, envs, info = O.find_groundstate(psi0, H, O.VUMPS(D=1, maxiter=200, tol=1e-10))
    assert abs(O.expectationvalue(psi, H, envs).real - (-7.0)) < 1e-10
