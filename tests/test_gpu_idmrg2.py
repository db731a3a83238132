"""Two-site IDMRG on the GPU against the oracle (src/algorithms/groundstates/idmrg.jl:90-235,
effective.jl:113-197): the two-site action, fixed-iteration trajectories with bond growth,
and converged energies."""
import math

import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,D", [(3, 6), (4, 16)])
def test_ac2_apply_matches_oracle(ctx, seed, D):
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    opsi = O.randomimps([2, 2], D=D, seed=seed)
    oenvs = O.build_envs(opsi, oH)
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = upload_envs(psi, H, oenvs)
    rng = np.random.default_rng(seed)
    for p in (0, 1):
        q = (p + 1) % 2
        x = (rng.standard_normal((D, 2, 2, D)) + 1j * rng.standard_normal((D, 2, 2, D))).astype(complex)
        y = imps.ac2_apply(envs, H, p + 1, x)
        yo = O.ac2_apply(oenvs.lefts[p], oH[p], oH[q], oenvs.rights[q], x)
        assert rel(y, yo) < 1e-13


def test_idmrg2_trajectory_with_bond_growth(ctx):
    # D grows 4 -> 8 at the first split; k sweeps with tol = 0 follow the oracle
    W = O.tfim_hamiltonian(J=1.0, h=1.5).Ws[0]
    oH = O.SchurMPO([W, W])
    H = to_device_mpo(oH)
    opsi0 = O.randomimps([2, 2], D=4, seed=43)
    psi0 = upload_state(ctx, opsi0)
    for k in (1, 3):
        psi, envs, info = imps.find_groundstate(psi0, H, imps.IDMRG2(D=8, maxiter=k, tol=0.0))
        opsi, oenvs, oinfo = O.idmrg2_groundstate(opsi0, oH, O.IDMRG2(D=8, maxiter=k, tol=0.0))
        assert psi.chi == [8, 8]
        e = imps.expectationvalue(psi, H, envs).real
        eo = O.expectationvalue(opsi, oH, oenvs).real
        assert abs(e - eo) < 1e-9
        np.testing.assert_allclose(info.losses[1:], oinfo["losses"][1:], rtol=1e-4, atol=1e-9)
        for b in (1, 2):
            np.testing.assert_allclose(imps.entanglement_spectrum(psi, b),
                                       O.entanglement_spectrum(opsi, b), atol=1e-9)


def test_idmrg2_converges_to_vumps_energy(ctx):
    W = O.tfim_hamiltonian(J=1.0, h=1.5).Ws[0]
    oH = O.SchurMPO([W, W])
    H = to_device_mpo(oH)
    psi, envs, info = imps.find_groundstate(imps.randomimps([2, 2], D=4, seed=7, ctx=ctx), H,
                                            imps.IDMRG2(D=12, maxiter=100, tol=1e-10))
    assert info.converged
    assert max(psi.chi) <= 12
    pv, ev, _ = imps.find_groundstate(imps.randomimps([2, 2], D=12, seed=8, ctx=ctx), H,
                                      imps.VUMPS(D=12, maxiter=300, tol=1e-10))
    assert abs(imps.expectationvalue(psi, H, envs).real - imps.expectationvalue(pv, H, ev).real) < 1e-8


def test_idmrg2_critical_heisenberg_energy(ctx):
    # the reference's anchor e0 = 1/4 - ln 2 (test/algorithms/idmrg.jl), within the D = 12 gap
    H = imps.SparseIMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi, envs, info = imps.find_groundstate(imps.randomimps([2, 2], D=12, seed=5, ctx=ctx), H,
                                            imps.IDMRG2(D=12, maxiter=200, tol=1e-9))
    e = imps.expectationvalue(psi, H, envs).real / 2
    assert abs(e - (0.25 - math.log(2.0))) < 2e-4


def test_idmrg2_rejects_one_site_cell(ctx):
    with pytest.raises(imps.ArgumentError):
        imps.find_groundstate(imps.randomimps([2], D=4, seed=1, ctx=ctx), imps.tfim_hamiltonian(),
                              imps.IDMRG2(D=4, maxiter=2))
