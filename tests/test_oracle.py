"""The CPU oracle against the reference's own known-answer tests (CPU only).

Each test names the reference test it restates.  These pin the oracle; the GPU
tests then compare the CUDA path against the oracle.
"""
import math

import numpy as np
import pytest

import oracle as O


def test_dynamictol_formula():
    # test/algorithms/api.jl:453-462
    bare = dict(tol=1.0e-8, maxiter=100)
    assert O.updatetol(bare, 5, 0.1) is bare
    dt = O.DynamicTol(bare, 1.0e-14, 1.0e-4, 0.1)
    assert math.isclose(O.updatetol(dt, 1, 5.0e-4)["tol"], 5.0e-5)
    assert O.updatetol(dt, 1, 5.0e-4)["maxiter"] == 100
    assert math.isclose(O.updatetol(dt, 1, 1.0e-20)["tol"], 1.0e-14)
    assert math.isclose(O.updatetol(dt, 1, 1.0e20)["tol"], 1.0e-4)
    with pytest.raises(ValueError):
        O.DynamicTol(bare, 1.0, 0.1, 0.1)


def test_defaults_match_reference():
    # src/utility.jl:308-320
    assert O.Defaults.D == 64 and O.Defaults.maxiter == 300 and O.Defaults.tolgauge == 1e-13
    assert O.Defaults.tol == 1e-10 and O.Defaults.krylovdim == 30
    assert (O.Defaults.tol_min, O.Defaults.tol_max) == (1e-14, 1e-4)
    assert (O.Defaults.eigs_tolfactor, O.Defaults.gauge_tolfactor, O.Defaults.envs_tolfactor) == (1e-3, 1e-6, 1e-4)


def test_linsolve_coefficients():
    # test/algorithms/api.jl:248-251: (a0 + a1 A) x = b with A = 2I -> 3x = b
    rng = np.random.default_rng(0)
    b = rng.standard_normal(5).astype(complex)
    x, info = O.gmres(lambda v: 2 * v, b, np.zeros(5, complex), 1e-12, 30, 300, 1.0, 1.0)
    assert info.converged
    np.testing.assert_allclose(x, b / 3, atol=1e-12)


def test_integrate_exact_diagonal():
    # test/algorithms/api.jl:469-478
    v0 = np.array([1.0 + 0j, 2.0])
    vr, info = O.exponentiate(lambda v: v, -1j * 0.1, v0, 1e-12, 30, 30)
    np.testing.assert_allclose(vr, np.exp(-1j * 0.1) * v0, atol=1e-13)
    vi, _ = O.exponentiate(lambda v: v, -0.1, v0, 1e-12, 30, 30)
    np.testing.assert_allclose(vi, np.exp(-0.1) * v0, atol=1e-13)


def test_regularize_trace_zero():
    # test/algorithms/api.jl:243-246
    rng = np.random.default_rng(1)
    M = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    M = O.regularize(M, np.eye(3), np.eye(3) / 3)
    assert abs(np.trace(M)) < 1e-12


def test_identity_heff_and_hermiticity():
    # test/algorithms/api.jl:226-239
    H = O.tfim_hamiltonian()
    psi = O.randomimps([2], D=4, seed=23)
    rng = np.random.default_rng(24)
    x = O.random_site_tensors([2], 4, 24)[0]
    I4 = np.eye(4, dtype=complex).reshape(4, 1, 4)
    Wid = np.eye(2, dtype=complex).reshape(1, 2, 1, 2)
    np.testing.assert_allclose(O.ac_apply(I4, Wid, I4, x), x, atol=1e-14)
    envs = O.build_envs(psi, H)
    y = O.random_site_tensors([2], 4, 25)[0]
    hac = lambda v: O.ac_apply(envs.lefts[0], H[0], envs.rights[0], v)
    assert abs(np.vdot(x, hac(y)) - np.vdot(hac(x), y)) < 1e-7
    c1 = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    c2 = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    hc = lambda v: O.c_apply(envs.lefts[0], envs.rights[0], v)
    assert abs(np.vdot(c1, hc(c2)) - np.vdot(hc(c1), c2)) < 1e-7


def test_contract_identity_expval():
    # test/algorithms/api.jl:253-257: identity MPO single-site contraction = ||AC||^2
    psi = O.randomimps([2], D=4, seed=23)
    I4 = np.eye(4, dtype=complex).reshape(4, 1, 4)
    Wid = np.eye(2, dtype=complex).reshape(1, 2, 1, 2)
    AC = psi.AC[0]
    assert abs(np.vdot(AC, O.ac_apply(I4, Wid, I4, AC)) - np.linalg.norm(AC) ** 2) < 1e-10


def test_canonical_relations_and_dot():
    psi = O.randomimps([2, 2], D=6, seed=7)
    for i in range(2):
        Dl, d, Dr = psi.AL[i].shape
        A2 = O.freshape(psi.AL[i], (Dl * d, Dr))
        np.testing.assert_allclose(A2.conj().T @ A2, np.eye(Dr), atol=1e-12)
        B = O.freshape(psi.AR[i], (Dl, d * Dr))
        np.testing.assert_allclose(B @ B.conj().T, np.eye(Dl), atol=1e-12)
        np.testing.assert_allclose(psi.AC[i], O._mulCA(psi.C[i - 1], psi.AR[i]), atol=1e-10)
    assert abs(O.state_dot(psi, psi) - 1) < 1e-10


def test_dot_between_states_and_product_state():
    # test/algorithms/api.jl:130-141 and test/states/mps.jl:1-44
    a = O.randomimps([2, 2], D=6, seed=11)
    b = O.randomimps([2, 2], D=6, seed=12)
    ab, ba = O.state_dot(a, b), O.state_dot(b, a)
    assert abs(ab) <= 1 + 1e-8
    assert abs(ab - np.conj(ba)) < 1e-8
    # product state |up, down>: norm 1 and <sigma_z> = +1 / -1
    ALs = []
    for k in (0, 1):
        A = O.fzeros((1, 2, 1))
        A[0, k, 0] = 1.0
        ALs.append(A)
    p = O.canonical_from_AL(ALs, np.eye(1, dtype=complex))
    assert abs(O.state_dot(p, p) - 1) < 1e-12
    assert abs(O.local_expectation1(p, 0, O.sigma("z")) - 1) < 1e-12
    assert abs(O.local_expectation1(p, 1, O.sigma("z")) + 1) < 1e-12


def test_gauge_fixes_from_random_tensors():
    # test/algorithms/api.jl:150-160: left, right and mixed gauge fixes of random tensors
    rng = np.random.default_rng(5)
    As = [np.asfortranarray(rng.standard_normal((6, 2, 6)) + 1j * rng.standard_normal((6, 2, 6))) for _ in range(2)]
    psi = O.canonical_from_sites(As)
    for l in range(2):
        A2 = O.freshape(psi.AL[l], (12, 6))
        assert np.linalg.norm(A2.conj().T @ A2 - np.eye(6)) < 1e-10
        B = O.freshape(psi.AR[l], (6, 12))
        assert np.linalg.norm(B @ B.conj().T - np.eye(6)) < 1e-10
    assert abs(np.linalg.norm(psi.AC[0]) - 1) < 1e-10


def test_qrpos_lqpos_positive():
    rng = np.random.default_rng(3)
    M = rng.standard_normal((12, 5)) + 1j * rng.standard_normal((12, 5))
    Q, R = O.qrpos(M)
    np.testing.assert_allclose(Q @ R, M, atol=1e-12)
    assert np.all(np.diag(R).real >= 0) and np.allclose(np.diag(R).imag, 0)
    Lf, Q2 = O.lqpos(M.T)
    np.testing.assert_allclose(Lf @ Q2, M.T, atol=1e-12)
    assert np.all(np.diag(Lf).real >= 0) and np.allclose(np.diag(Lf).imag, 0)


def test_regauge_reconstructs():
    # test/algorithms/api.jl:170-174 (regauge! consistency): at a fixed point AC = AL C
    psi = O.randomimps([2], D=5, seed=9)
    AL = O.regauge(psi.AC[0], psi.C[0])
    np.testing.assert_allclose(O._mulAL(AL, psi.C[0]), psi.AC[0], atol=1e-9)


def test_tfim_n1_vumps_galerkin():
    # test/algorithms/api.jl:481-489: N=1 TFIM, D=10, tol 1e-11 -> Galerkin < 1e-9,
    # calc_galerkin == info.itererr; plus e0 = -4/pi at finite-D tolerance
    H = O.tfim_hamiltonian()
    psi0 = O.randomimps([2], D=10, seed=41)
    psi, envs, info = O.find_groundstate(psi0, H, O.VUMPS(D=10, maxiter=300, tol=1e-11))
    assert info["itererr"] < 1e-9
    assert O.calc_galerkin(psi, H, envs) == info["itererr"]
    e = O.expectationvalue(psi, H, envs).real
    assert abs(e + 4 / math.pi) < 1e-5


def test_xxz_vumps_energy():
    # test/algorithms/vumps.jl:4-12: XXZ Delta=1, N=2, D=12 -> |e - (1/4 - ln 2)| < 2e-4
    H = O.heisenberg_hamiltonian()
    psi0 = O.randomimps([2, 2], D=12, seed=2)
    psi, envs, info = O.find_groundstate(psi0, H, O.VUMPS(D=12, maxiter=300, tol=1e-10))
    e = O.expectationvalue(psi, H, envs).real / 2
    assert info["itererr"] < 1e-9
    assert abs(e - (0.25 - math.log(2))) < 2e-4


def test_tdvp_conservation():
    # test/algorithms/tdvp.jl:14-24 (short version): real time conserves energy and norm
    H = O.heisenberg_hamiltonian()
    psi0 = O.randomimps([2, 2], D=8, seed=5)
    psi, envs, _ = O.find_groundstate(psi0, H, O.VUMPS(D=8, maxiter=200, tol=1e-9))
    e0 = O.expectationvalue(psi, H, envs).real / 2
    ts = [-1j * 0.01 * k for k in range(6)]
    pt, et, hist = O.time_evolve(psi, H, ts)
    assert abs(hist[-1].real / 2 - e0) < 1e-6
    assert abs(np.linalg.norm(pt.AC[0]) - 1) < 1e-8


def test_hubbard_model_hermitian_and_anchor():
    H = O.hubbard_hamiltonian()
    W = H[0]
    h2 = sum(np.kron(W[0, :, k, :], W[k, :, 5, :]) for k in range(1, 5))
    assert np.linalg.norm(h2 - h2.conj().T) < 1e-14
    # the Lieb-Wu anchor and the TFIM anchor used by the energy checks
    assert abs(O.hubbard_e0() - (-2.5737293678984)) < 1e-9
    assert abs(O.tfim_e0() + 4 / math.pi) < 1e-12


def _open_chain_from_mpo(W, L):
    """Hamiltonian of an open chain of L sites from a Schur MPO site tensor W (m, d, n, d):
    first level at the left end, last level at the right end."""
    m, d = W.shape[0], W.shape[1]
    X = [np.eye(1, dtype=complex) if k == 0 else None for k in range(m)]
    for _ in range(L):
        Y = [None] * m
        for a in range(m):
            if X[a] is None:
                continue
            for b in range(m):
                blk = W[a, :, b, :]
                if np.any(blk):
                    t = np.kron(X[a], blk)
                    Y[b] = t if Y[b] is None else Y[b] + t
        X = Y
    return X[m - 1]


def test_hubbard_mpo_open_chain_exact_diagonalisation():
    # the w = 6 Jordan-Wigner Hubbard MPO against an independent second-quantised build on an
    # open chain of 4 sites (8 fermionic modes, 256 states): identical spectra
    t, U, mu, L = 1.0, 4.0, 2.0, 4
    Hm = _open_chain_from_mpo(O.hubbard_hamiltonian()[0], L)
    nm = 2 * L
    a = np.array([[0, 1], [0, 0]], dtype=complex)     # annihilates the occupied state |1>
    z = np.diag([1.0, -1.0]).astype(complex)
    eye = np.eye(2, dtype=complex)

    def mode_op(k):
        ops = [z] * k + [a] + [eye] * (nm - k - 1)
        out = ops[0]
        for o in ops[1:]:
            out = np.kron(out, o)
        return out
    c = [mode_op(k) for k in range(nm)]           # mode 2 i + s: site i, spin s
    n = [ck.conj().T @ ck for ck in c]
    Hf = np.zeros((2 ** nm, 2 ** nm), dtype=complex)
    for i in range(L - 1):
        for s in range(2):
            hop = c[2 * i + s].conj().T @ c[2 * (i + 1) + s]
            Hf += -t * (hop + hop.conj().T)
    for i in range(L):
        Hf += U * n[2 * i] @ n[2 * i + 1] - mu * (n[2 * i] + n[2 * i + 1])
    assert np.linalg.norm(Hm - Hm.conj().T) < 1e-12
    em = np.linalg.eigvalsh(Hm)
    ef = np.linalg.eigvalsh(Hf)
    assert np.max(np.abs(em - ef)) < 1e-10
