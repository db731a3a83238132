"""Parity of the CUDA path with the oracle at the benchmark configurations' own sizes.

* TFIM J=h=1, N=1, D=16, seed 1 (the plain FP64 configuration): VUMPS to Galerkin
  1e-10 on the GPU and through the oracle from the same seeded site tensors; the
  converged energies agree to 1e-10 and sit at the finite-D distance from -4/pi.
* XXZ Jxy=Jz=1, N=2, D=256, seed 2: one environment build (DMRGCache) against the
  oracle's, the AC and C effective Hamiltonians on it to 1e-12, and a two-iteration
  fixed-count VUMPS trajectory (tol = 0) to 1e-10 in energy.
* Hubbard (JW, t=1, U=4, mu=2), N=2, D=1024: one FP64 AC and C apply against the
  oracle's at <= 1e-11 relative, and the int8-split apply within its accuracy bound.

Round-off grows with D, so these pin the FP64 bars at the sizes the benchmark runs.
"""
import math

import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
import oracle as O
from gpu_helpers import rel, to_device_mpo, upload_envs, upload_state

pytestmark = pytest.mark.gpu


def test_tfim_d16_seed1_converges_like_the_oracle(ctx):
    As = O.random_site_tensors([2], 16, 1)
    oH = O.tfim_hamiltonian()
    opsi, oenvs, oinfo = O.find_groundstate(O.canonical_from_sites(As), oH, O.VUMPS(D=16, maxiter=300, tol=1e-10))
    eo = O.expectationvalue(opsi, oH, oenvs).real
    H = imps.tfim_hamiltonian()
    psi0 = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
    psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=16, maxiter=300, tol=1e-10))
    e = imps.expectationvalue(psi, H, envs).real
    assert oinfo["converged"] and info.converged
    assert info.itererr <= 1e-10
    assert abs(e - eo) < 1e-10
    # finite-D distance from the exact energy density -4/pi (1.6e-7 at D=16)
    assert abs(e + 4 / math.pi) < 1e-6


@pytest.fixture(scope="module")
def xxz256():
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    opsi = O.canonical_from_sites(O.random_site_tensors([2, 2], 256, 2))
    oenvs = O.build_envs(opsi, oH)
    return oH, opsi, oenvs


def test_xxz_d256_envs_and_heff(ctx, xxz256):
    oH, opsi, oenvs = xxz256
    H = to_device_mpo(oH)
    psi = upload_state(ctx, opsi)
    envs = imps.DMRGCache(psi, H)
    for l in range(2):
        assert rel(envs.leftenv(l + 1), oenvs.lefts[l]) < 1e-9
        assert rel(envs.rightenv(l + 1), oenvs.rights[l]) < 1e-9
    # effective Hamiltonians on identical environments: pure contraction round-off
    envs_o = upload_envs(psi, H, oenvs)
    rng = np.random.default_rng(22)
    for site in (1, 2):
        x = rng.standard_normal((256, 2, 256)) + 1j * rng.standard_normal((256, 2, 256))
        y = imps.AC_hamiltonian(site, psi, H, psi, envs_o)(x)
        yo = O.ac_apply(oenvs.lefts[site - 1], oH[site - 1], oenvs.rights[site - 1], x)
        assert rel(y, yo) < 1e-12
        c = rng.standard_normal((256, 256)) + 1j * rng.standard_normal((256, 256))
        yc = imps.C_hamiltonian(site, psi, H, psi, envs_o)(c)
        yco = O.c_apply(oenvs.lefts[site % 2], oenvs.rights[site - 1], c)
        assert rel(yc, yco) < 1e-12


def test_xxz_d256_two_iteration_trajectory(ctx, xxz256):
    oH, opsi, oenvs = xxz256
    H = to_device_mpo(oH)
    psi0 = upload_state(ctx, opsi)
    psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=256, maxiter=2, tol=0.0))
    po, eo_envs, oinfo = O.find_groundstate(opsi, oH, O.VUMPS(D=256, maxiter=2, tol=0.0), envs=oenvs)
    e = imps.expectationvalue(psi, H, envs).real
    eo = O.expectationvalue(po, oH, eo_envs).real
    assert abs(e - eo) < 1e-10 * max(1.0, abs(eo))
    np.testing.assert_allclose(info.losses, oinfo["losses"], rtol=1e-5)


@pytest.fixture(scope="module")
def hubbard1024():
    D = 1024
    W = O.hubbard_hamiltonian().Ws[0]
    rng = np.random.default_rng(3)

    def rc(*s):
        return np.asfortranarray(rng.standard_normal(s) + 1j * rng.standard_normal(s))
    GL, GR, GL2 = rc(D, 6, D), rc(D, 6, D), rc(D, 6, D)
    x, c = rc(D, 4, D), rc(D, D)
    y_ac = O.ac_apply(GL, W, GR, x)
    y_c = O.c_apply(GL2, GR, c)
    return W, GL, GR, GL2, x, c, y_ac, y_c


def _hubbard_apply(ctx, case):
    W, GL, GR, GL2, x, c, _, _ = case
    H = imps.SparseIMPO([W, W])
    psi = imps.CanonicalIMPS(ctx, [4, 4], [1024, 1024])
    envs = imps.DMRGCache(psi, H, build=False)
    envs.set_leftenv(1, GL)
    envs.set_rightenv(1, GR)
    envs.set_leftenv(2, GL2)
    y = imps.AC_hamiltonian(1, psi, H, psi, envs)(x)
    yc = imps.C_hamiltonian(1, psi, H, psi, envs)(c)
    return y, yc


def test_hubbard_d1024_fp64_heff(ctx, hubbard1024):
    y, yc = _hubbard_apply(ctx, hubbard1024)
    assert rel(y, hubbard1024[6]) <= 1e-11
    assert rel(yc, hubbard1024[7]) <= 1e-11


@pytest.mark.parametrize("s,bound", [(4, 1e-6), (5, 2e-8), (6, 1e-10)])
def test_hubbard_d1024_split_heff(hubbard1024, s, bound):
    # each split GEMM truncates both operands below 2^-7s of their row / column
    # scales (per-element bound 2 K (s+2) 2^-7s r_i c_j); on these O(1) random
    # operands the relative Frobenius error of the whole AC / C apply sits about two
    # orders below that bound, so these bars leave a 10x margin on what it measures
    cs = imps.Context(0)
    cs.set_precision(L.IMPS_PREC_SPLIT_I8, s)
    y, yc = _hubbard_apply(cs, hubbard1024)
    assert rel(y, hubbard1024[6]) <= bound
    assert rel(yc, hubbard1024[7]) <= bound
    cs.close()
