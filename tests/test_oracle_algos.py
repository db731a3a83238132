"""Oracle IDMRG and imaginary-time TDVP against the reference's known answers
(CPU only): test/algorithms/idmrg.jl:1-23 and test/algorithms/tdvp.jl:27-34."""
import math

import numpy as np
import pytest

import oracle as O

E_XXZ = 0.25 - math.log(2.0)


def test_idmrg_xxz_matches_exact_and_vumps():
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    pv, ev_envs, _ = O.find_groundstate(O.randomimps([2, 2], D=12, seed=31), H, O.VUMPS(D=12, maxiter=300, tol=1e-10))
    ev = O.expectationvalue(pv, H, ev_envs).real / 2
    pi, ei_envs, _ = O.idmrg_groundstate(O.randomimps([2, 2], D=12, seed=32), H, O.IDMRG(D=12, maxiter=300, tol=1e-9))
    ei = O.expectationvalue(pi, H, ei_envs).real / 2
    assert abs(ei - E_XXZ) < 2e-4
    assert abs(ei - ev) < 2e-4
    p8, e8_envs, _ = O.idmrg_groundstate(O.randomimps([2, 2], D=8, seed=33), H, O.IDMRG(D=8, maxiter=300, tol=1e-9))
    assert max(a.shape[2] for a in p8.AL) <= 8
    assert abs(O.expectationvalue(p8, H, e8_envs).real / 2 - E_XXZ) < 1e-3


def test_imaginary_time_tdvp_reaches_ground_state():
    # exp(-H beta) with steps of 0.05 up to beta = 20 at D = 8: within 2e-3 of the
    # infinite-chain energy (the finite-D gap is ~1e-3)
    H = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi0 = O.randomimps([2, 2], D=8, seed=34)
    tspan = [-0.05 * k for k in range(401)]
    psi, envs, _ = O.time_evolve(psi0, H, tspan, O.TDVP(), observer=lambda p, k, t: 0.0)
    e = O.expectationvalue(psi, H, O.build_envs(psi, H)).real / 2
    assert abs(e - E_XXZ) < 2e-3


def test_idmrg2_gapped_tfim_grows_bond_and_matches_vumps():
    # two-site IDMRG grows D = 4 -> 8 (truncdim(8)) and reaches the VUMPS fixed point;
    # src/algorithms/groundstates/idmrg.jl:90-235
    W = O.tfim_hamiltonian(J=1.0, h=1.5).Ws[0]
    H = O.SchurMPO([W, W])
    p2, envs2, info = O.idmrg2_groundstate(O.randomimps([2, 2], D=4, seed=43), H, O.IDMRG2(D=8, maxiter=100, tol=1e-10))
    assert info["converged"]
    assert [a.shape for a in p2.AL] == [(8, 2, 8), (8, 2, 8)]
    pv, envv, _ = O.find_groundstate(O.randomimps([2, 2], D=8, seed=44), H, O.VUMPS(D=8, maxiter=300, tol=1e-10))
    e2 = O.expectationvalue(p2, H, envs2).real / 2
    ev = O.expectationvalue(pv, H, envv).real / 2
    assert abs(e2 - ev) < 1e-9


def test_idmrg2_critical_tfim_energy():
    # TFIM at h = J: e0 = -4/pi (the reference's twosite test anchor); D = 8 is within 1e-5
    W = O.tfim_hamiltonian(J=1.0, h=1.0).Ws[0]
    H = O.SchurMPO([W, W])
    p2, envs2, info = O.idmrg2_groundstate(O.randomimps([2, 2], D=8, seed=41), H, O.IDMRG2(D=8, maxiter=100, tol=1e-9))
    assert max(a.shape[2] for a in p2.AL) <= 8
    assert info["losses"][-1] < info["losses"][1]
    assert abs(O.expectationvalue(p2, H, envs2).real / 2 + 4 / math.pi) < 1e-5


def test_idmrg2_requires_two_site_cell():
    with pytest.raises(ValueError):
        O.idmrg2_groundstate(O.randomimps([2], D=4, seed=1), O.tfim_hamiltonian(), O.IDMRG2(D=4, maxiter=2))
