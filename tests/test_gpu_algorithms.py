"""End-to-end algorithms on the GPU: VUMPS, TDVP, IDMRG against the oracle and
against the reference's own analytic anchors."""
import math

import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_state

pytestmark = pytest.mark.gpu


def test_vumps_tfim_n1_reference_kat(ctx):
    # test/algorithms/api.jl:481-489: N=1 TFIM D=10 tol 1e-11 -> Galerkin < 1e-9,
    # calc_galerkin == info.itererr; e within finite-D tolerance of -4/pi
    H = imps.tfim_hamiltonian()
    psi0 = imps.randomimps([2], D=10, seed=41, ctx=ctx)
    psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=10, maxiter=300, tol=1e-11))
    assert info.converged and info.itererr < 1e-9
    assert imps.calc_galerkin(psi, H, envs) == info.itererr
    e = imps.expectationvalue(psi, H, envs).real
    assert abs(e + 4 / math.pi) < 1e-5
    # same seeded start through the oracle: same converged energy (FP64 vs FP64: 1e-10)
    opsi, oenvs, oinfo = O.find_groundstate(O.randomimps([2], D=10, seed=41), O.tfim_hamiltonian(),
                                            O.VUMPS(D=10, maxiter=300, tol=1e-11))
    assert abs(e - O.expectationvalue(opsi, O.tfim_hamiltonian(), oenvs).real) < 1e-10


def test_vumps_fixed_iterations_trajectory(ctx):
    # groundstate_concordance protocol: k iterations with tol = 0, compare energy and Galerkin
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    H = to_device_mpo(oH)
    opsi0 = O.randomimps([2, 2], D=8, seed=21)
    psi0 = upload_state(ctx, opsi0)
    for k in (1, 3):
        psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=8, maxiter=k, tol=0.0))
        opsi, oenvs, oinfo = O.find_groundstate(opsi0, oH, O.VUMPS(D=8, maxiter=k, tol=0.0))
        e = imps.expectationvalue(psi, H, envs)
        eo = O.expectationvalue(opsi, oH, oenvs)
        assert abs(e - eo) < 1e-10 * max(1, abs(eo))
        np.testing.assert_allclose(info.losses, oinfo["losses"], rtol=1e-6, atol=1e-12)


def test_vumps_xxz_reference_kat(ctx):
    # test/algorithms/vumps.jl:4-12
    H = imps.SparseIMPO([imps.heisenberg_hamiltonian().Ws[0]] * 2)
    psi0 = imps.randomimps([2, 2], D=12, seed=2, ctx=ctx)
    psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=12, maxiter=300, tol=1e-10))
    e = imps.expectationvalue(psi, H, envs).real / 2
    assert info.itererr < 1e-9
    assert abs(e - (0.25 - math.log(2))) < 2e-4


def test_vumps_iter_abi_matches_python_loop(ctx):
    # imps_vumps_iter (one C call per iteration) == the Python mirror of vumps.jl
    oH = O.tfim_hamiltonian()
    H = to_device_mpo(oH)
    opsi0 = O.randomimps([2], D=12, seed=31)
    psi_a = upload_state(ctx, opsi0)
    envs_a = imps.DMRGCache(psi_a, H)
    eps = imps.calc_galerkin(psi_a, H, envs_a)
    imps.recalculate(envs_a, psi_a, H, tol=imps.updatetol(imps.Defaults.alg_environments(), 0, eps)["tol"])
    lib = L.load()
    out = []
    for it in (1, 2, 3):
        info = L.VumpsInfo()
        assert lib.imps_vumps_iter(envs_a.h, H.handle(ctx), psi_a.h, it, eps, info) == 0
        eps = info.galerkin
        out.append((info.galerkin, info.energy_re))
    psi_b, envs_b, ib = imps.find_groundstate(upload_state(ctx, opsi0), H, imps.VUMPS(D=12, maxiter=3, tol=0.0))
    assert abs(out[-1][0] - ib.losses[-1]) < 1e-9
    assert abs(out[-1][1] - imps.expectationvalue(psi_b, H, envs_b).real) < 1e-10


def test_tdvp_conservation_and_oracle(ctx):
    # test/algorithms/tdvp.jl:14-24 (shortened) and trajectory parity with the oracle
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    H = to_device_mpo(oH)
    opsi, oenvs, _ = O.find_groundstate(O.randomimps([2, 2], D=8, seed=5), oH, O.VUMPS(D=8, maxiter=200, tol=1e-9))
    psi = upload_state(ctx, opsi)
    e0 = O.expectationvalue(opsi, oH, oenvs).real / 2
    ts = [-1j * 0.01 * k for k in range(6)]
    pt, et, hist = imps.time_evolve(psi, H, ts)
    assert len(hist) == 6
    assert abs(hist[-1].real / 2 - e0) < 1e-6
    assert abs(pt.norm() - 1) < 1e-8
    opt, oet, ohist = O.time_evolve(opsi, oH, ts)
    np.testing.assert_allclose(np.real(hist), np.real(ohist), atol=1e-10)


def test_tdvp_quench_local_observable(ctx):
    # quench protocol at small size: TFIM h=0.5 ground state evolved under h=1.5
    oH0 = O.tfim_hamiltonian(h=0.5)
    oH1 = O.tfim_hamiltonian(h=1.5)
    opsi, _, _ = O.find_groundstate(O.randomimps([2], D=8, seed=4), oH0, O.VUMPS(D=8, maxiter=100, tol=1e-10))
    psi = upload_state(ctx, opsi)
    H1 = to_device_mpo(oH1)
    sx = O.sigma("x")
    envs = imps.DMRGCache(psi, H1)
    oenvs = O.build_envs(opsi, oH1)
    for k in range(3):
        psi, envs = imps.timestep(psi, H1, -0.01j, imps.TDVP(), envs)
        opsi, oenvs = O.timestep(opsi, oH1, -0.01j, O.TDVP(), oenvs)
        assert abs(imps.expectationvalue(psi, ((1,), sx)) - O.local_expectation1(opsi, 0, sx)) < 1e-8


def test_idmrg_sweeps_match_oracle(ctx):
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    H = to_device_mpo(oH)
    opsi0 = O.randomimps([2, 2], D=8, seed=6)
    psi, envs, info = imps.find_groundstate(upload_state(ctx, opsi0), H, imps.IDMRG(D=8, maxiter=4, tol=0.0))
    opsi, oenvs, oinfo = O.idmrg_groundstate(opsi0, oH, O.IDMRG(D=8, maxiter=4, tol=0.0))
    e = imps.expectationvalue(psi, H, envs).real
    eo = O.expectationvalue(opsi, oH, oenvs).real
    assert abs(e - eo) < 1e-8
    np.testing.assert_allclose(info.losses[1:], oinfo["losses"][1:], rtol=1e-5, atol=1e-10)


def test_local_expval_and_dot(ctx):
    opsi = O.randomimps([2, 2], D=6, seed=13)
    psi = upload_state(ctx, opsi)
    for site in (1, 2):
        for op in (O.sigma("x"), O.sigma("z")):
            assert abs(imps.expectationvalue(psi, ((site,), op)) - O.local_expectation1(opsi, site - 1, op)) < 1e-12
    assert abs(psi.dot() - O.state_dot(opsi, opsi)) < 1e-12
