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
