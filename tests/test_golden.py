"""The oracle against the committed golden fixtures and the reference's analytic anchors (CPU only).

``tests/golden/make_golden.py`` wrote the fixtures; this file recomputes each of
them with the oracle, so a change in the oracle's arithmetic shows up here
before it can move the GPU parity tests."""
import json
import math
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def test_heff_fixture():
    g = load("heff_hubbard_n2.npz")
    for s in range(2):
        assert rel(O.ac_apply(g[f"GL{s}"], g["W"], g[f"GR{s}"], g[f"x{s}"]), g[f"yac{s}"]) < 1e-13
        assert rel(O.c_apply(g[f"GL{(s + 1) % 2}"], g[f"GR{s}"], g[f"c{s}"]), g[f"yc{s}"]) < 1e-13


def test_heff_fixture_is_hubbard_mpo():
    g = load("heff_hubbard_n2.npz")
    assert np.array_equal(g["W"], O.hubbard_hamiltonian().Ws[0])


def test_pushes_fixture():
    g = load("pushes_xxz.npz")
    assert rel(O.push_env_left(g["Lm"], g["A"], g["B"]), g["left_id"]) < 1e-13
    assert rel(O.push_env_right(g["Rm"], g["A"], g["B"]), g["right_id"]) < 1e-13
    assert rel(O.push_mpo_left(g["Lw"], g["W"], g["A"]), g["left_mpo"]) < 1e-13
    assert rel(O.push_mpo_right(g["Rw"], g["W"], g["A"]), g["right_mpo"]) < 1e-13


def test_qrpos_fixture():
    g = load("qrpos.npz")
    Q, R = O.qrpos(g["M"])
    assert rel(Q, g["Q"]) < 1e-12 and rel(R, g["R"]) < 1e-12
    Lf, Qr = O.lqpos(g["Mt"])
    assert rel(Lf, g["L"]) < 1e-12 and rel(Qr, g["Qr"]) < 1e-12
    assert rel(O.regauge(g["AC"], g["C"]), g["AL"]) < 1e-12
    assert np.all(np.diag(g["R"]).real >= 0) and np.allclose(np.diag(g["R"]).imag, 0)


def test_vumps_trajectory_fixture():
    g = load("vumps_xxz_n2.npz")
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi0 = O.CanonicalIMPS([g["AL0"], g["AL1"]], [g["AR0"], g["AR1"]], [g["C0"], g["C1"]], [g["AC0"], g["AC1"]])
    psi, envs, info = O.find_groundstate(psi0, oH, O.VUMPS(D=8, maxiter=1, tol=0.0))
    assert abs(O.expectationvalue(psi, oH, envs) - g["energy_k1"]) < 1e-12
    np.testing.assert_allclose(info["losses"], g["losses_k1"], rtol=1e-9)


def test_reference_kats_json():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        k = json.load(f)
    assert math.isclose(k["tfim_e0_critical"]["value"], O.tfim_e0(1.0, 1.0), rel_tol=1e-12)
    assert math.isclose(k["xxz_e0"]["value"], 0.25 - math.log(2.0))
    dt = O.DynamicTol(dict(tol=1e-8, maxiter=100), k["dynamictol"]["tol_min"], k["dynamictol"]["tol_max"],
                      k["dynamictol"]["tol_factor"])
    for eps, want in k["dynamictol"]["cases"]:
        assert math.isclose(O.updatetol(dt, 1, eps)["tol"], want)
    for v in k.values():
        assert "source" in v and ".jl:" in v["source"]
