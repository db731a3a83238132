"""Batched VUMPS (imps_vumps_iter_batch): independent TFIM instances with uneven
bond dimensions, each on its own context and stream, against the same
instances solved one at a time and against the exact TFIM energy."""
import math

import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps

pytestmark = pytest.mark.gpu


def tfim_e0(h, J=1.0):
    from scipy.integrate import quad
    return -quad(lambda k: math.sqrt(J * J + h * h - 2 * J * h * math.cos(k)), 0, math.pi)[0] / math.pi


def test_batch_matches_sequential_and_exact():
    hs = [0.6, 0.8, 1.2, 1.4]
    Ds = [8, 12, 16, 24]
    ctxs = [imps.Context(0) for _ in hs]
    try:
        Hs = [imps.tfim_hamiltonian(1.0, h) for h in hs]
        psi0s = [imps.CanonicalIMPS.from_sites(imps.random_site_tensors([2], D, 1000 + k), ctx=c)
                 for k, (D, c) in enumerate(zip(Ds, ctxs))]
        alg = imps.VUMPS(maxiter=200, tol=1e-10)
        out = imps.find_groundstate_batch(psi0s, Hs, alg, nthreads=4)
        for k, (psi, envs, info) in enumerate(out):
            assert info.converged and info.itererr <= 1e-10
            e = imps.expectationvalue(psi, Hs[k], envs).real
            # the same instance alone, through the per-instance driver
            psi_s, envs_s, info_s = imps.find_groundstate(psi0s[k], Hs[k], alg)
            e_s = imps.expectationvalue(psi_s, Hs[k], envs_s).real
            assert abs(e - e_s) < 1e-10
            assert abs(e - tfim_e0(hs[k])) < 1e-5
            # fixed-state coupling gradient == Hellmann-Feynman <dH/dh> = -<sigma_z>
            dW = [(imps.tfim_hamiltonian(1.0, hs[k] + 1e-3).Ws[0] - imps.tfim_hamiltonian(1.0, hs[k] - 1e-3).Ws[0]) / 2e-3]
            g = imps.coupling_gradient(psi, Hs[k], dW, envs).real
            assert abs(g + imps.expectationvalue(psi, (1, imps.sigma("z"))).real) < 1e-9
    finally:
        for c in ctxs:
            c.close()


def test_batch_shared_context_runs_in_order(ctx):
    Hs = [imps.tfim_hamiltonian(1.0, 0.7), imps.tfim_hamiltonian(1.0, 1.3)]
    psi0s = [imps.CanonicalIMPS.from_sites(imps.random_site_tensors([2], 8, 7 + k), ctx=ctx) for k in range(2)]
    out = imps.find_groundstate_batch(psi0s, Hs, imps.VUMPS(maxiter=100, tol=1e-9), nthreads=8)
    for k, (psi, envs, info) in enumerate(out):
        assert info.converged
        psi_s, envs_s, _ = imps.find_groundstate(psi0s[k], Hs[k], imps.VUMPS(maxiter=100, tol=1e-9))
        assert abs(imps.expectationvalue(psi, Hs[k], envs) - imps.expectationvalue(psi_s, Hs[k], envs_s)) < 1e-10
