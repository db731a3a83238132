"""Generate the golden fixtures under ``tests/golden/`` from the CPU oracle.

Run from the repository root: ``python tests/golden/make_golden.py``.

The reference (Julia + KrylovKit + FMA) cannot run in this environment, so the
fixtures are frozen outputs of the oracle on seeded inputs (NumPy PCG64); the
oracle itself is pinned to the reference's known-answer tests, which are stored
beside them in ``reference_kats.json`` with the reference test file:line each
one comes from.  ``tests/test_golden.py`` recomputes every fixture with the
oracle (CPU) and checks the analytic anchors; ``tests/test_gpu_golden.py``
checks the CUDA path against the same files.

Fixtures (all column-major complex128, shapes as in the reference):
  heff_hubbard_n2.npz  AC / C effective-Hamiltonian actions, Hubbard JW (d=4, w=6), N=2, D=12
  pushes_xxz.npz       identity and MPO transfer pushes, XXZ (d=2, w=5), Dl=9, Dr=7
  qrpos.npz            QRpos / LQpos / regauge factors
  vumps_xxz_n2.npz     VUMPS trajectory (k = 1, 3 iterations, tol = 0), XXZ N=2 D=8, seed 21
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def rc(rng, *shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def heff_fixture():
    rng = np.random.default_rng(1201)
    D, N = 12, 2
    W = O.hubbard_hamiltonian().Ws[0]
    w, d = W.shape[0], W.shape[1]
    GL = [rc(rng, D, w, D) for _ in range(N)]
    GR = [rc(rng, D, w, D) for _ in range(N)]
    out = dict(W=W)
    for s in range(N):
        x = rc(rng, D, d, D)
        c = rc(rng, D, D)
        out[f"GL{s}"], out[f"GR{s}"] = GL[s], GR[s]
        out[f"x{s}"], out[f"c{s}"] = x, c
        out[f"yac{s}"] = O.ac_apply(GL[s], W, GR[s], x)
        # C_hamiltonian at bond s uses leftenv(s + 1) and rightenv(s)
        out[f"yc{s}"] = O.c_apply(GL[(s + 1) % N], GR[s], c)
    return out


def pushes_fixture():
    rng = np.random.default_rng(1202)
    Dl, Dr = 9, 7
    W = O.heisenberg_hamiltonian().Ws[0]
    w, d = W.shape[0], W.shape[1]
    A, B = rc(rng, Dl, d, Dr), rc(rng, Dl, d, Dr)
    Lm, Rm = rc(rng, Dl, Dl), rc(rng, Dr, Dr)
    Lw, Rw = rc(rng, Dl, w, Dl), rc(rng, Dr, w, Dr)
    return dict(W=W, A=A, B=B, Lm=Lm, Rm=Rm, Lw=Lw, Rw=Rw,
                left_id=O.push_env_left(Lm, A, B), right_id=O.push_env_right(Rm, A, B),
                left_mpo=O.push_mpo_left(Lw, W, A), right_mpo=O.push_mpo_right(Rw, W, A))


def qr_fixture():
    rng = np.random.default_rng(1203)
    M = rc(rng, 20, 9)
    Mt = rc(rng, 9, 20)
    Q, R = O.qrpos(M)
    Lf, Qr = O.lqpos(Mt)
    AC, C = rc(rng, 6, 3, 6), rc(rng, 6, 6)
    return dict(M=M, Q=Q, R=R, Mt=Mt, L=Lf, Qr=Qr, AC=AC, C=C, AL=O.regauge(AC, C))


def vumps_fixture():
    oH = O.SchurMPO([O.heisenberg_hamiltonian().Ws[0]] * 2)
    psi0 = O.randomimps([2, 2], D=8, seed=21)
    out = {}
    for l in range(2):
        out[f"AL{l}"], out[f"AR{l}"] = psi0.AL[l], psi0.AR[l]
        out[f"C{l}"], out[f"AC{l}"] = psi0.C[l], psi0.AC[l]
    for k in (1, 3):
        psi, envs, info = O.find_groundstate(psi0, oH, O.VUMPS(D=8, maxiter=k, tol=0.0))
        out[f"energy_k{k}"] = np.array(O.expectationvalue(psi, oH, envs))
        out[f"losses_k{k}"] = np.array(info["losses"])
    return out


def reference_kats():
    """Analytic anchors and tolerances from the reference's own tests (file:line)."""
    return {
        "tfim_e0_critical": {"value": -4.0 / math.pi, "source": "test/algorithms/vumps.jl:14-18; README.md:58",
                             "check": "|e/N + 4/pi| < 1e-6 at D=12, N=2, tol 1e-10"},
        "xxz_e0": {"value": 0.25 - math.log(2.0), "source": "test/algorithms/vumps.jl:4-12",
                   "check": "|e/N - (1/4 - ln 2)| < 2e-4 at D=12, N=2, tol 1e-10; itererr < 1e-9"},
        "tfim_n1_galerkin": {"value": 1e-9, "source": "test/algorithms/api.jl:481-489",
                             "check": "N=1 TFIM D=10 tol 1e-11: Galerkin < 1e-9 and calc_galerkin == itererr"},
        "tdvp_conservation": {"energy_tol": 1e-6, "norm_tol": 1e-8, "source": "test/algorithms/tdvp.jl:14-24"},
        "linsolve_2I": {"a0": 1.0, "a1": 1.0, "diag": 2.0, "source": "test/algorithms/api.jl:248-251",
                        "check": "(a0 + a1 A) x = b with A = 2I gives x = b / 3"},
        "regularize_trace_zero": {"source": "test/algorithms/api.jl:243-246"},
        "dynamictol": {"source": "test/algorithms/api.jl:453-462",
                       "cases": [[5.0e-4, 5.0e-5], [1.0e-20, 1.0e-14], [1.0e20, 1.0e-4]],
                       "tol_min": 1.0e-14, "tol_max": 1.0e-4, "tol_factor": 0.1},
    }


def main():
    np.savez_compressed(os.path.join(HERE, "heff_hubbard_n2.npz"), **heff_fixture())
    np.savez_compressed(os.path.join(HERE, "pushes_xxz.npz"), **pushes_fixture())
    np.savez_compressed(os.path.join(HERE, "qrpos.npz"), **qr_fixture())
    np.savez_compressed(os.path.join(HERE, "vumps_xxz_n2.npz"), **vumps_fixture())
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(reference_kats(), f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
