"""Non-uniform bond and physical dimensions on the CUDA path, against the oracle
(the CPU side is tests/test_oracle_nonuniform.py), after the reference's
test/algorithms/envs.jl:30-126: environments and energy on a unit cell with bond
profile [2, 4, 2]; invariance of the energy under zero-padding of one bond (to
1e-10); a unit cell with physical dimensions [2, 3, 2] (norm, local identities,
the energy shift of on-site identities); and the product ground state E = -7 of
diagonal on-site fields found by VUMPS."""
import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_state
from test_oracle_nonuniform import pad_bond, tfim_cell

pytestmark = pytest.mark.gpu


def _profile_state(rng, chi, d=2):
    N = len(chi)
    ALs = []
    for l in range(N):
        dl, dr = chi[(l - 1) % N], chi[l]
        M = rng.standard_normal((dl * d, dr)) + 1j * rng.standard_normal((dl * d, dr))
        q, _ = np.linalg.qr(M)
        ALs.append(O.freshape(np.asfortranarray(q[:, :dr]), (dl, d, dr)))
    return O.canonical_from_AL(ALs, np.eye(chi[N - 1], dtype=complex))


def test_profile_242_envs_and_energy(ctx):
    opsi = _profile_state(np.random.default_rng(7), [2, 4, 2])
    oH = tfim_cell(1.0, 1.3, 3)
    oenvs = O.build_envs(opsi, oH)
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = imps.DMRGCache(psi, H)
    for l in range(3):
        assert envs.leftenv(l + 1).shape == oenvs.lefts[l].shape
        assert envs.rightenv(l + 1).shape == oenvs.rights[l].shape
        assert rel(envs.leftenv(l + 1), oenvs.lefts[l]) < 1e-9
        assert rel(envs.rightenv(l + 1), oenvs.rights[l]) < 1e-9
    e = imps.expectationvalue(psi, H, envs)
    eo = O.expectationvalue(opsi, oH, oenvs)
    assert abs(e - eo) < 1e-10
    assert abs(imps.calc_galerkin(psi, H, envs) - O.calc_galerkin(opsi, oH, oenvs)) < 1e-9


def test_zero_padding_leaves_gpu_energy_unchanged(ctx):
    # test/algorithms/envs.jl:61-66 on the device: |E_padded - E| < 1e-10
    oH = tfim_cell(1.0, 1.3, 3)
    H = to_device_mpo(oH)
    opsi = O.randomimps([2, 2, 2], D=4, seed=13)
    psp = pad_bond(opsi, 1, 1, np.random.default_rng(3))
    psi = upload_state(ctx, opsi)
    pp = upload_state(ctx, psp)
    E0 = imps.expectationvalue(psi, H, imps.DMRGCache(psi, H)).real
    Ep = imps.expectationvalue(pp, H, imps.DMRGCache(pp, H)).real
    assert abs(Ep - E0) < 1e-10
    assert abs(E0 - O.expectationvalue(opsi, oH, O.build_envs(opsi, oH)).real) < 1e-10


def test_heterogeneous_physical_dims(ctx):
    # test/algorithms/envs.jl:75-126: d = [2, 3, 2] from a seeded random start
    dims = [2, 3, 2]
    As = O.random_site_tensors(dims, 4, 3)
    psi = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
    opsi = O.canonical_from_sites(As)
    assert abs(abs(psi.dot()) - 1) < 1e-10
    for l, d in enumerate(dims):
        assert abs(imps.expectationvalue(psi, (l + 1, np.eye(d))).real - 1) < 1e-10
        assert rel(psi.AC[l + 1], opsi.AC[l]) < 1e-8
    rng = np.random.default_rng(3)
    hd = []
    for d in dims:
        h = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        hd.append((h + h.conj().T) / 2)
    H = imps.SparseIMPO([imps.mpohamiltonian(h, []) for h in hd])
    Hs = imps.SparseIMPO([imps.mpohamiltonian(h + np.eye(h.shape[0]), []) for h in hd])
    e0 = imps.expectationvalue(psi, H, imps.DMRGCache(psi, H)).real
    e1 = imps.expectationvalue(psi, Hs, imps.DMRGCache(psi, Hs)).real
    oH = O.SchurMPO([O.mpohamiltonian(h, []) for h in hd])
    assert abs(e0 - O.expectationvalue(opsi, oH, O.build_envs(opsi, oH)).real) < 1e-10
    assert abs(e1 - e0 - 3.0) < 1e-10


def test_heterogeneous_product_ground_state(ctx):
    lams = [np.array([-2.0, 1.0]), np.array([-3.0, 0.0, 2.0]), np.array([-2.0, 1.0])]
    H = imps.SparseIMPO([imps.mpohamiltonian(np.diag(l).astype(complex), []) for l in lams])
    ALs = []
    for l in lams:
        A = np.zeros((1, len(l), 1), dtype=complex, order="F")
        A[0, int(np.argmin(l)), 0] = 1.0
        ALs.append(A)
    psi0 = imps.CanonicalIMPS.from_AL(ALs, np.eye(1, dtype=complex), ctx=ctx)
    psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=1, maxiter=200, tol=1e-10))
    assert abs(imps.expectationvalue(psi, H, envs).real - (-7.0)) < 1e-10
