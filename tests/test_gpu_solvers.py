"""Krylov solvers, gauge fixing and environment builds on the GPU against the oracle
(identical algorithms, so agreement is to accumulated FP64 round-off)."""
import math

import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
import oracle as O
from gpu_helpers import phase_fix, rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu


def test_linsolve_diag_kat(ctx):
    # test/algorithms/api.jl:248-251: A = 2I, (1 + 1 A) x = b -> x = b/3
    rng = np.random.default_rng(0)
    b = rng.standard_normal(5).astype(complex)
    x, info = imps.linsolve(2 * np.ones(5), b, np.zeros(5), 1.0, 1.0, tol=1e-12)
    np.testing.assert_allclose(x, b / 3, atol=1e-12)
    assert info.converged == 1


def test_linsolve_diag_matches_oracle(ctx):
    rng = np.random.default_rng(1)
    n = 200
    dv = 0.5 + rng.random(n) + 0.1j * rng.standard_normal(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    # well-conditioned: |1 - 0.3 dv| >= 0.55
    x, info = imps.linsolve(dv, b, np.zeros(n), 1.0, -0.3, tol=1e-11, krylovdim=12)
    xr, ir = O.gmres(lambda v: dv * v, b, np.zeros(n, complex), 1e-11, 12, 300, 1.0, -0.3)
    assert rel(x, xr) < 1e-9
    assert info.numops == ir.numops and info.numiter == ir.numiter


def test_exponentiate_diag_kat(ctx):
    # test/algorithms/api.jl:469-478
    lib = L.load()
    v0 = np.array([1.0 + 0j, 2.0])
    out = np.zeros(2, complex)
    info = L.KrylovInfo()
    d = np.ones(2, complex)
    for dt in (-1j * 0.1, -0.1):
        st = lib.imps_exponentiate_diag(ctx.h, 2, L.dptr(d), dt.real if isinstance(dt, complex) else dt,
                                        dt.imag if isinstance(dt, complex) else 0.0, L.dptr(v0), L.dptr(out),
                                        1e-12, 30, 30, None)
        assert st == 0
        np.testing.assert_allclose(out, np.exp(dt) * v0, atol=1e-13)


def test_canonicalize_matches_oracle(ctx):
    As = O.random_site_tensors([2, 2], 8, 11)
    opsi = O.canonical_from_sites(As)
    psi = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
    for l in range(2):
        assert rel(psi.AL[l + 1], opsi.AL[l]) < 1e-9
        assert rel(psi.AR[l + 1], opsi.AR[l]) < 1e-9
        assert rel(psi.C[l + 1], opsi.C[l]) < 1e-9
        assert rel(psi.AC[l + 1], opsi.AC[l]) < 1e-9
    assert abs(psi.dot() - 1) < 1e-10


@pytest.mark.parametrize("model,dims,D,seed", [("tfim", [2], 12, 3), ("xxz", [2, 2], 10, 4),
                                               ("hubbard", [4, 4], 6, 5)])
def test_env_build_and_observables(ctx, model, dims, D, seed):
    oH = {"tfim": O.tfim_hamiltonian, "xxz": O.heisenberg_hamiltonian, "hubbard": O.hubbard_hamiltonian}[model]()
    oH = O.SchurMPO([oH.Ws[0]] * len(dims))
    opsi = O.randomimps(dims, D=D, seed=seed)
    oenvs = O.build_envs(opsi, oH)
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = imps.DMRGCache(psi, H)
    for l in range(len(dims)):
        assert rel(envs.leftenv(l + 1), oenvs.lefts[l]) < 1e-8
        assert rel(envs.rightenv(l + 1), oenvs.rights[l]) < 1e-8
    assert abs(imps.calc_galerkin(psi, H, envs) - O.calc_galerkin(opsi, oH, oenvs)) < 1e-9
    e = imps.expectationvalue(psi, H, envs)
    eo = O.expectationvalue(opsi, oH, oenvs)
    assert abs(e - eo) < 1e-9 * max(1, abs(eo))
    # warm rebuild gives the same environments
    imps.recalculate(envs, psi, H, tol=1e-12)
    oenvs2 = O.build_envs(opsi, oH, tol=1e-12, init=oenvs)
    for l in range(len(dims)):
        assert rel(envs.leftenv(l + 1), oenvs2.lefts[l]) < 1e-8


def test_eigsolve_ac_c(ctx):
    oH = O.heisenberg_hamiltonian()
    oH = O.SchurMPO([oH.Ws[0]] * 2)
    opsi = O.randomimps([2, 2], D=10, seed=8)
    oenvs = O.build_envs(opsi, oH)
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = upload_envs(psi, H, oenvs)
    alg = dict(tol=1e-10, krylovdim=30, maxiter=300, eager=True)
    lam, v = imps.fixedpoint(imps.AC_hamiltonian(1, psi, H, psi, envs), opsi.AC[0], "SR", alg)
    lr, vr, _ = O.lanczos_eigsolve(lambda x: O.ac_apply(oenvs.lefts[0], oH[0], oenvs.rights[0], x), opsi.AC[0],
                                   1e-10, 30, 300, True)
    assert abs(lam - lr) < 1e-9 * max(1, abs(lr))
    assert rel(v, vr) < 1e-6
    lam, v = imps.fixedpoint(imps.C_hamiltonian(1, psi, H, psi, envs), opsi.C[0], "SR", alg)
    lr, vr, _ = O.lanczos_eigsolve(lambda x: O.c_apply(oenvs.lefts[1], oenvs.rights[0], x), opsi.C[0], 1e-10, 30,
                                   300, True)
    assert abs(lam - lr) < 1e-9 * max(1, abs(lr))
    assert rel(v, vr) < 1e-6


def test_exponentiate_ac(ctx):
    oH = O.heisenberg_hamiltonian()
    opsi = O.randomimps([2], D=8, seed=12)
    oenvs = O.build_envs(opsi, oH)
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = upload_envs(psi, H, oenvs)
    x = imps.integrate(imps.AC_hamiltonian(1, psi, H, psi, envs), opsi.AC[0], -0.05j)
    xr, _ = O.exponentiate(lambda v: O.ac_apply(oenvs.lefts[0], oH[0], oenvs.rights[0], v), -0.05j, opsi.AC[0],
                           1e-10, 30, 300)
    assert rel(x, xr) < 1e-9
    assert abs(np.linalg.norm(x) - np.linalg.norm(opsi.AC[0])) < 1e-9
