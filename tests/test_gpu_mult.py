"""MPO application mult(W, psi, VOMPS) on the GPU against the oracle
(src/algorithms/arithmetics/mult.jl, arithmetics/envs.jl:51-93, transfermatrix.jl:77-107):
the initial guess, the ternary fixed points through the local maps, and whole runs."""
import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
import oracle as O
from gpu_helpers import rel, upload_state

pytestmark = pytest.mark.gpu


def _tfim_gs(D, seed):
    H0 = O.tfim_hamiltonian(J=1.0, h=0.5)
    psi, _, _ = O.find_groundstate(O.randomimps([2], D=D, seed=seed), H0, O.VUMPS(D=D, maxiter=200, tol=1e-10))
    return psi


@pytest.mark.parametrize("N", [2, 3])
def test_guess_matches_oracle(ctx, N):
    # N >= 2 only: with one site the guess identifies the left and right bond bases of two
    # different SVDs (compress.jl:183-188, "an approximation for the initial guess"), so it
    # depends on the SVD's phase convention; only the converged mult result is unique
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * N)
    opsi = O.randomimps([2] * N, D=6, seed=8)
    W = O.timeevompo(H, -1j * 0.02, "WII")
    ox = O.canonical_from_sites(O.svdguess_mult_sites(W, opsi.AL, 7))
    x = imps.svdguess_mult(imps.DenseIMPO(W), upload_state(ctx, opsi), 7)
    assert x.chi == [a.shape[2] for a in ox.AL]
    for b in range(1, N + 1):
        np.testing.assert_allclose(imps.entanglement_spectrum(x, b), O.entanglement_spectrum(ox, b), atol=1e-10)


def test_ternary_fixed_points_local_maps(ctx):
    # bra and ket of different bond dimensions, a two-site cell and a dense MPO
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    W = O.timeevompo(H, -1j * 0.05, "WII")
    obra = O.randomimps([2, 2], D=5, seed=11)
    oket = O.randomimps([2, 2], D=7, seed=12)
    GLs, GRs = O.mixed_fixedpoints(obra, W, oket, 1e-12, 300)
    oenv = O.MultCache(W, obra, oket, GLs, GRs)
    bra, ket = upload_state(ctx, obra), upload_state(ctx, oket)
    envs = imps.MultCache(bra, imps.DenseIMPO(W), ket, tol=1e-12)
    for l in range(2):
        ac, c = envs.local_maps(l + 1)
        assert rel(ac, O.mult_local_ac(oenv, l)) < 1e-9
        assert rel(c, O.mult_local_c(oenv, l)) < 1e-9
        # each GR has unit norm (the normalisation convention)
        assert abs(np.linalg.norm(envs.rightenv(l + 1)) - 1) < 1e-12
    assert abs(envs.galerkin() - O.mult_galerkin(oenv, obra)) < 1e-9


def test_mult_wii_step_matches_oracle_and_tdvp(ctx):
    opsi = _tfim_gs(8, 4)
    H1 = O.tfim_hamiltonian(J=1.0, h=1.5)
    W = O.timeevompo(H1, -1j * 0.01, "WII")
    y, envs, info = imps.mult(imps.DenseIMPO(W), upload_state(ctx, opsi), imps.VOMPS(D=8, maxiter=50, tol=1e-10))
    oy, oenvs, oinfo = O.mult(W, opsi, O.VOMPS(D=8, maxiter=50, tol=1e-10))
    assert info.converged and info.itererr <= 1e-10 and oinfo["converged"]
    assert abs(abs(O.state_dot(oy, _download(y))) - 1) < 1e-10
    sx = O.sigma("x")
    e_gpu = imps.expectationvalue(y, ((1,), sx))
    assert abs(e_gpu - O.local_expectation1(oy, 0, sx)) < 1e-9
    p1, _ = O.timestep(opsi, H1, -0.01j, O.TDVP(), O.build_envs(opsi, H1))
    assert abs(e_gpu - O.local_expectation1(p1, 0, sx)) < 1e-6


def test_mult_identity_two_site_cell(ctx):
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    opsi, _, _ = O.find_groundstate(O.randomimps([2, 2], D=6, seed=21), H, O.VUMPS(D=6, maxiter=200, tol=1e-9))
    psi = upload_state(ctx, opsi)
    y, envs, info = imps.mult(imps.identityimpo([2, 2]), psi, imps.VOMPS(D=6, maxiter=30, tol=1e-10))
    assert info.converged
    assert abs(abs(O.state_dot(opsi, _download(y))) - 1) < 1e-10


def _download(psi):
    N = len(psi)
    return O.CanonicalIMPS(list(psi.AL), list(psi.AR), list(psi.C), list(psi.AC))


def test_mult_lossless_bond_equals_naive_product(ctx):
    # test/algorithms/arithmetics.jl:290-297 on the device: at the lossless bond dimension
    # mult returns the naive product W . psi
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    W = O.timeevompo(H, -0.05j, "WII")
    opsi = O.randomimps([2, 2], D=3, seed=9)
    As = []
    for l in range(2):
        wl, u, wr, _ = W[l].shape
        bl, _, br = opsi.AL[l].shape
        B5 = np.einsum("wurd,bdc->wburc", W[l], opsi.AL[l])
        As.append(np.asfortranarray(B5.reshape((wl * bl, u, wr * br), order="F")))
    ref = O.canonical_from_sites(As)
    y, _, info = imps.mult(imps.DenseIMPO(W), upload_state(ctx, opsi), imps.VOMPS(D=12, maxiter=300, tol=1e-10))
    assert max(y.chi) == 12
    assert abs(O.state_dot(_download(y), ref)) > 1 - 1e-8
