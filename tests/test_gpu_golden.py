"""The CUDA path against the committed golden fixtures (FP64; 1e-12 relative for
single contractions, the oracle trajectory tolerances for VUMPS)."""
import os

import numpy as np
import pytest

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L
from gpu_helpers import rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_heff_golden(ctx):
    g = load("heff_hubbard_n2.npz")
    N, D = 2, g["x0"].shape[0]
    d = g["W"].shape[1]
    H = imps.SparseIMPO([g["W"]] * N)
    psi = imps.CanonicalIMPS(ctx, [d] * N, [D] * N)
    envs = imps.DMRGCache(psi, H, build=False)
    for s in range(N):
        envs.set_leftenv(s + 1, g[f"GL{s}"])
        envs.set_rightenv(s + 1, g[f"GR{s}"])
    for s in range(N):
        assert rel(imps.AC_hamiltonian(s + 1, psi, H, psi, envs)(g[f"x{s}"]), g[f"yac{s}"]) < 1e-12
        assert rel(imps.C_hamiltonian(s + 1, psi, H, psi, envs)(g[f"c{s}"]), g[f"yc{s}"]) < 1e-12


def test_pushes_golden(ctx):
    g = load("pushes_xxz.npz")
    H = imps.SparseIMPO([g["W"]])
    assert rel(imps.push_env_left(g["Lm"], g["A"], g["B"], ctx=ctx), g["left_id"]) < 1e-12
    assert rel(imps.push_env_right(g["Rm"], g["A"], g["B"], ctx=ctx), g["right_id"]) < 1e-12
    assert rel(imps.push_mpo_left(g["Lw"], H, 1, g["A"], ctx=ctx), g["left_mpo"]) < 1e-12
    assert rel(imps.push_mpo_right(g["Rw"], H, 1, g["A"], ctx=ctx), g["right_mpo"]) < 1e-12


def test_qrpos_golden(ctx):
    g = load("qrpos.npz")
    Q, R = imps.qrpos(g["M"], ctx=ctx)
    assert rel(Q, g["Q"]) < 1e-12 and rel(R, g["R"]) < 1e-12
    Lf, Qr = imps.lqpos(g["Mt"], ctx=ctx)
    assert rel(Lf, g["L"]) < 1e-12 and rel(Qr, g["Qr"]) < 1e-12
    assert rel(imps.regauge(g["AC"], g["C"], ctx=ctx), g["AL"]) < 1e-12


def test_vumps_trajectory_golden(ctx):
    g = load("vumps_xxz_n2.npz")
    W = imps.heisenberg_hamiltonian()
    H = imps.SparseIMPO([W.Ws[0]] * 2)
    psi0 = imps.CanonicalIMPS(ctx, [2, 2], [8, 8])
    for l in range(2):
        psi0.set(L.IMPS_AL, l, g[f"AL{l}"])
        psi0.set(L.IMPS_AR, l, g[f"AR{l}"])
        psi0.set(L.IMPS_C, l, g[f"C{l}"])
        psi0.set(L.IMPS_AC, l, g[f"AC{l}"])
    for k in (1, 3):
        psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=8, maxiter=k, tol=0.0))
        e = imps.expectationvalue(psi, H, envs)
        assert abs(e - g[f"energy_k{k}"]) < 1e-10 * max(1.0, abs(g[f"energy_k{k}"]))
        np.testing.assert_allclose(info.losses, g[f"losses_k{k}"], rtol=1e-6, atol=1e-12)
