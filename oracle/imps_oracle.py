"""NumPy/SciPy restatement of the InfiniteMPSAlgorithms VUMPS/TDVP inner loop.

TEST INFRASTRUCTURE ONLY -- the oracle.  It is imported by ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``, and by
nothing that ships.  The product path (``infinitempsalgorithms_b200``) never
calls it.

Parity status
-------------
* The reference is pure Julia and cannot run in this container (no ``julia``,
  and its dependencies KrylovKit / TensorOperations / FiniteMPSAlgorithms are
  absent).  Every function below restates the cited reference lines.
* Pinned against the reference's own known-answer tests (``tests/test_oracle.py``):
  TFIM ``e0 = -4/pi`` (``test/algorithms/vumps.jl:15-18``), XXZ
  ``e0 = 1/4 - ln 2`` (``test/algorithms/vumps.jl:7-12``), the N=1 TFIM Galerkin < 1e-9 run
  (``test/algorithms/api.jl:481-489``), Heff Hermiticity and identity
  (``api.jl:226-239``), ``regularize!`` (``api.jl:243-246``), ``linsolve``
  coefficients (``api.jl:248-251``), ``contract_mpo_expval``
  (``api.jl:253-257``), ``DynamicTol`` (``api.jl:453-462``), ``integrate``
  (``api.jl:469-478``) and the TDVP conservation laws (``test/algorithms/tdvp.jl:14-24``).
* KrylovKit internals (restart policy, Ritz-vector phase) are UNPINNED: the
  library is absent.  The Krylov solvers below restate the published
  algorithms (thick-restart Lanczos, restarted GMRES with Givens rotations,
  Krylov exponential with sub-stepping, Arnoldi with Ritz restart); the CUDA
  runtime implements exactly the same algorithms, so the trajectories agree.

Conventions (identical to the reference, Julia column-major)
-------------------------------------------------------------
* site tensors ``A[a, s, b]`` of shape ``(Dl, d, Dr)``;
* left environments ``GL[bra, level, ket]``, right ``GR[ket, level, bra]``
  (``src/algorithms/groundstates/effective.jl:3-5``);
* dense MPO tensors ``W[wl, u, wr, s]`` with ``u`` the output (bra) leg
  (``envs.jl:332``, ``tompotensor``);
* all arrays are kept in Fortran order and reshaped with ``order='F'`` so each
  reshape is the reference's ``reshape``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

__all__ = [
    "freshape", "fzeros", "C128", "energy_grad_mpo", "energy_grad_al", "Defaults", "DynamicTol", "alg_eigsolve", "alg_gauge",
    "alg_environments", "alg_expsolve", "canonical_from_AL", "canonical_from_sites",
    "canonical_from_AL_keepAL", "_mulAL", "_mulCA", "hubbard_operators", "updatetol", "sigma", "spin", "mpohamiltonian",
    "SchurMPO", "tfim_hamiltonian", "heisenberg_hamiltonian", "hubbard_hamiltonian",
    "tfim_e0", "hubbard_e0", "qrpos", "lqpos", "lanczos_eigsolve", "gmres",
    "exponentiate", "arnoldi_dominant", "KrylovInfo", "push_env_left",
    "push_env_right", "push_slice_left", "push_slice_right", "push_mpo_left",
    "push_mpo_right", "regularize", "CanonicalIMPS", "uniform_leftorth",
    "uniform_rightorth", "gaugefix", "regauge", "randomimps", "random_site_tensors",
    "state_dot", "DMRGCache", "build_envs", "ac_apply", "c_apply", "calc_galerkin",
    "expectationvalue", "local_expectation1", "VUMPS", "TDVP", "IDMRG",
    "find_groundstate", "vumps_iteration", "timestep", "time_evolve", "idmrg_groundstate",
    "dominant_env", "normalize_envs", "build_envs_dense", "expectationvalue_dense", "apply_local", "correlator",
    "entanglement_spectrum", "renyi_entropy", "entropy",
    "timeevompo", "timeevompo_site", "mpo_ring",
    "IDMRG2", "ac2_apply", "VOMPS", "MultCache", "push_ternary_left", "push_ternary_right", "mult_ac",
    "mult_c", "env_start_vector", "mixed_fixedpoints", "mult_galerkin", "svdguess_mult_sites", "mult_sweeps",
    "mult_local_ac", "mult_local_c",
    "mult", "ac2", "idmrg2_split", "idmrg2_sweep", "idmrg2_groundstate",
]

C128 = np.complex128


def freshape(x, shape):
    return np.reshape(x, shape, order="F")


def fzeros(shape, dtype=C128):
    return np.zeros(shape, dtype=dtype, order="F")


# --------------------------------------------------------------------------
# Defaults and DynamicTol  (src/utility.jl:136-171, 297-365)
# --------------------------------------------------------------------------
class Defaults:
    """Mirror of ``module Defaults`` (``src/utility.jl:297-365``)."""
    D = 64
    maxiter = 300
    tolgauge = 1.0e-13
    tol = 1.0e-10
    verbosity = 0
    krylovdim = 30
    dynamic_tols = True
    tol_min = 1.0e-14
    tol_max = 1.0e-4
    eigs_tolfactor = 1.0e-3
    gauge_tolfactor = 1.0e-6
    envs_tolfactor = 1.0e-4


@dataclass
class DynamicTol:
    """``DynamicTol(alg, tol_min, tol_max, tol_factor)`` (``src/utility.jl:136-148``).

    ``alg`` is a dict with at least ``tol`` and ``maxiter``.
    """
    alg: dict
    tol_min: float = 1.0e-6
    tol_max: float = 1.0e-2
    tol_factor: float = 0.1

    def __post_init__(self):
        if not (0 <= self.tol_min <= self.tol_max):
            raise ValueError("DynamicTol requires 0 <= tol_min <= tol_max")


def updatetol(alg, it: int, eps: float):
    """``updatetol`` (``src/utility.jl:151-157``): clamp(eps*f/sqrt(iter), min, max)."""
    if not isinstance(alg, DynamicTol):
        return alg
    it = max(it, 1)
    new_tol = min(max(eps * alg.tol_factor / math.sqrt(it), alg.tol_min), alg.tol_max)
    out = dict(alg.alg)
    out["tol"] = new_tol
    return out


def alg_eigsolve(tol=Defaults.tol, maxiter=Defaults.maxiter, krylovdim=Defaults.krylovdim,
                 eager=True, tol_factor=Defaults.eigs_tolfactor, dynamic=True):
    """``Defaults.alg_eigsolve`` (``src/utility.jl:330-340``)."""
    alg = dict(tol=tol, maxiter=maxiter, krylovdim=krylovdim, eager=eager)
    return DynamicTol(alg, Defaults.tol_min, Defaults.tol_max, tol_factor) if dynamic else alg


def alg_gauge(tol=Defaults.tolgauge, maxiter=Defaults.maxiter, dynamic=True):
    """``Defaults.alg_gauge`` (``src/utility.jl:349-353``)."""
    alg = dict(tol=tol, maxiter=maxiter)
    return DynamicTol(alg, Defaults.tol_min, Defaults.tol_max, Defaults.gauge_tolfactor) if dynamic else alg


def alg_environments(tol=Defaults.tol, maxiter=Defaults.maxiter, dynamic=True):
    """``Defaults.alg_environments`` (``src/utility.jl:358-364``)."""
    alg = dict(tol=tol, maxiter=maxiter)
    return DynamicTol(alg, Defaults.tol_min, Defaults.tol_max, Defaults.envs_tolfactor) if dynamic else alg


def alg_expsolve(tol=Defaults.tol, maxiter=Defaults.maxiter, krylovdim=Defaults.krylovdim):
    """``Defaults.alg_expsolve`` (``src/utility.jl:343-347``)."""
    return dict(tol=tol, maxiter=maxiter, krylovdim=krylovdim)


# --------------------------------------------------------------------------
# Models  (src/models.jl:61-122; Hubbard: own Jordan-Wigner construction)
# --------------------------------------------------------------------------
def sigma(which: str) -> np.ndarray:
    """Pauli matrices (``src/models.jl:64-66``)."""
    return {
        "x": np.array([[0, 1], [1, 0]], dtype=C128),
        "y": np.array([[0, -1j], [1j, 0]], dtype=C128),
        "z": np.array([[1, 0], [0, -1]], dtype=C128),
    }[which]


def spin(which: str) -> np.ndarray:
    """Spin-1/2 operators ``S = sigma/2`` (``src/models.jl:67-69``)."""
    return sigma(which) / 2


@dataclass
class SchurMPO:
    """A ``SparseIMPO`` (``src/operators/mpohamiltonian.jl:33-52``) as dense site tensors.

    ``Ws[l]`` has shape ``(m, d, n, d)`` = ``tompotensor(H[l])`` (``envs.jl:332``):
    ``W[i, u, j, s]`` is the ``(u_out, s_in)`` block from left level ``i`` to
    right level ``j``; a structurally missing block is all zeros.
    """
    Ws: List[np.ndarray]

    def __post_init__(self):
        N = len(self.Ws)
        if N == 0:
            raise ValueError("Ws must not be empty")
        for l in range(N):
            l1 = (l + 1) % N
            if self.Ws[l].shape[2] != self.Ws[l1].shape[0]:
                raise ValueError("level chain mismatch")  # mpohamiltonian.jl:58-67
        self.Ws = [np.asfortranarray(W, dtype=C128) for W in self.Ws]

    def __len__(self):
        return len(self.Ws)

    def __getitem__(self, l):
        return self.Ws[l % len(self.Ws)]

    def space_l(self, l):
        return self[l].shape[0]

    def space_r(self, l):
        return self[l].shape[2]

    def block(self, l, i, j):
        return self[l][i, :, j, :]

    def isidentitylevel(self, i: int, atol=1e-14) -> bool:
        """``isidentitylevel`` (``mpohamiltonian.jl:100-109``); ``i`` is 1-based."""
        if i == 1:
            return True
        for W in self.Ws:
            m, n = W.shape[0], W.shape[2]
            if i == m == n:
                continue
            if i > m - 1 or i > n - 1:
                return False
            blk = W[i - 1, :, i - 1, :]
            # isapprox(block, one(block); atol) with rtol = 0: Frobenius distance
            if np.linalg.norm(blk - np.eye(blk.shape[0])) > atol:
                return False
        return True

    def isemptylevel(self, i: int) -> bool:
        """``isemptylevel`` (``mpohamiltonian.jl:122-133``); ``i`` is 1-based."""
        if i == 1:
            return False
        if any(i == W.shape[2] for W in self.Ws):
            return False
        for W in self.Ws:
            m, n = W.shape[0], W.shape[2]
            dz = (i > m - 1 or i > n - 1) or not np.any(W[i - 1, :, i - 1, :])
            cz = (i > n - 1) or not np.any(W[0, :, i - 1, :])
            bz = (i > m - 1) or not np.any(W[i - 1, :, n - 1, :])
            if not (dz and cz and bz):
                return False
        return True


def mpohamiltonian(h1: np.ndarray, pairs: Sequence) -> np.ndarray:
    """Schur level matrix -> dense ``(n, d, n, d)`` tensor (``src/models.jl:82-100``).

    Levels 1 and n carry the identity, ``[1, n] = h1``, ``[1, k+1] = coeff_k a_k``
    and ``[k+1, n] = b_k``; all other blocks are missing (zero).
    """
    d = h1.shape[0]
    n = len(pairs) + 2
    W = fzeros((n, d, n, d))
    eye = np.eye(d, dtype=C128)
    W[0, :, 0, :] = eye
    W[n - 1, :, n - 1, :] = eye
    W[0, :, n - 1, :] = h1
    for k, (coeff, a, b) in enumerate(pairs):
        W[0, :, k + 1, :] = coeff * np.asarray(a, dtype=C128)
        W[k + 1, :, n - 1, :] = np.asarray(b, dtype=C128)
    return W


def tfim_hamiltonian(J=1.0, h=1.0) -> SchurMPO:
    """``H = -J sum sx sx - h sum sz`` (``src/models.jl:119-122``), w = 3."""
    return SchurMPO([mpohamiltonian(-h * sigma("z"), [(-J, sigma("x"), sigma("x"))])])


def heisenberg_hamiltonian(J=1.0, Delta=1.0, h=0.0) -> SchurMPO:
    """``H = J sum (SxSx + SySy + Delta SzSz) - h sum Sz`` (``src/models.jl:107-111``), w = 5."""
    Sx, Sy, Sz = spin("x"), spin("y"), spin("z")
    return SchurMPO([mpohamiltonian(-h * Sz, [(J, Sx, Sx), (J, Sy, Sy), (J * Delta, Sz, Sz)])])


def hubbard_operators():
    """Local fermion operators on ``(|0>, |up>, |dn>, |updn>)``, ``|updn> = c+_up c+_dn |0>``.

    Returns ``(c_up, c_dn, P, n, n_updn)`` with ``P = (-1)^n`` the local parity.
    """
    c_up = np.zeros((4, 4), dtype=C128)
    c_dn = np.zeros((4, 4), dtype=C128)
    c_up[0, 1] = 1.0   # c_up |up>   = |0>
    c_up[2, 3] = 1.0   # c_up |updn> = +|dn>
    c_dn[0, 2] = 1.0   # c_dn |dn>   = |0>
    c_dn[1, 3] = -1.0  # c_dn |updn> = -|up>
    P = np.diag([1.0, -1.0, -1.0, 1.0]).astype(C128)
    n = np.diag([0.0, 1.0, 1.0, 2.0]).astype(C128)
    n_updn = np.diag([0.0, 0.0, 0.0, 1.0]).astype(C128)
    return c_up, c_dn, P, n, n_updn


def hubbard_hamiltonian(t=1.0, U=4.0, mu=2.0) -> SchurMPO:
    """Spinful Hubbard chain via Jordan-Wigner, w = 6, built with ``mpohamiltonian``.

    ``H = -t sum_s (c+_{s,i} c_{s,i+1} + h.c.) + U sum n_up n_dn - mu sum n``.
    With ``c_{s,i} = (prod_{j<i} P_j) c_s`` the two hopping directions are
    ``(c+_s P) (x) c_s`` and ``(P c_s) (x) c+_s``, giving four channels.  The
    reference's own ``fermi_hubbard`` (``src/models.jl:164-178``) has only two
    channels and a non-Hermitian bond term, so it is not used.
    """
    c_up, c_dn, P, n, n_updn = hubbard_operators()
    h1 = U * n_updn - mu * n
    pairs = [
        (-t, c_up.conj().T @ P, c_up),
        (-t, P @ c_up, c_up.conj().T),
        (-t, c_dn.conj().T @ P, c_dn),
        (-t, P @ c_dn, c_dn.conj().T),
    ]
    return SchurMPO([mpohamiltonian(h1, pairs)])


def tfim_e0(J=1.0, h=1.0) -> float:
    """Exact TFIM ground-state energy density ``-(1/pi) int_0^pi sqrt(J^2+h^2-2Jh cos k) dk``."""
    from scipy.integrate import quad
    v, _ = quad(lambda k: math.sqrt(J * J + h * h - 2 * J * h * math.cos(k)), 0, math.pi, limit=200)
    return -v / math.pi


def hubbard_e0(t=1.0, U=4.0, mu=2.0) -> float:
    """Lieb-Wu half-filling energy per site minus ``mu * <n>`` (``<n> = 1``)."""
    from scipy.integrate import quad
    from scipy.special import j0, j1

    def f(w):
        x = w * U / (2 * t)
        if x > 700:
            return 0.0
        return j0(w) * j1(w) / (w * (1.0 + math.exp(x)))

    v, _ = quad(f, 0, np.inf, limit=500)
    return -4 * t * v - mu


# --------------------------------------------------------------------------
# QRpos / LQpos  (FiniteMPSAlgorithms leftorth/rightorth with QRpos/LQpos;
# usage: src/states/ortho.jl:150-153, 188-191, 214-227)
# --------------------------------------------------------------------------
def qrpos(M: np.ndarray):
    """``leftorth(M; alg = QRpos())``: ``M = Q R`` with a non-negative real diagonal of R."""
    Q, R = np.linalg.qr(M, mode="reduced")
    dg = np.diag(R)
    mag = np.abs(dg)
    ph = np.where(mag > 0, dg / np.where(mag > 0, mag, 1), 1.0)
    Q = Q * ph[None, :]
    R = R * np.conj(ph)[:, None]
    return np.asfortranarray(Q), np.asfortranarray(R)


def lqpos(M: np.ndarray):
    """``rightorth(M; alg = LQpos())``: ``M = L Q`` with a non-negative real diagonal of L."""
    Qp, Rp = qrpos(M.conj().T)
    return np.asfortranarray(Rp.conj().T), np.asfortranarray(Qp.conj().T)


# --------------------------------------------------------------------------
# Krylov solvers (KrylovKit restated; see the module docstring)
# --------------------------------------------------------------------------
@dataclass
class KrylovInfo:
    converged: int = 0
    numiter: int = 0
    numops: int = 0
    normres: float = float("nan")


class _KBasis:
    """Krylov basis stored as the leading columns of one preallocated column-major
    ``n x cap`` array (the projections are BLAS matrix-vector products on a view;
    no copy of the basis per step)."""

    def __init__(self, n: int, cap: int, v0: Optional[np.ndarray] = None):
        self.B = np.empty((n, cap), dtype=C128, order="F")
        self.m = 0
        if v0 is not None:
            self.append(v0)

    def append(self, v):
        self.B[:, self.m] = v
        self.m += 1

    def __len__(self):
        return self.m

    def __getitem__(self, k):
        return self.B[:, k]

    def mat(self, m: Optional[int] = None) -> np.ndarray:
        return self.B[:, : (self.m if m is None else m)]

    def reset(self, cols: np.ndarray):
        """Replace the basis by the columns of ``cols`` (n x k)."""
        k = cols.shape[1]
        self.B[:, :k] = cols
        self.m = k


def _cgs2(V: "_KBasis", w: np.ndarray):
    """Classical Gram-Schmidt with iterative refinement (KrylovKit's
    ``ClassicalGramSchmidtIR`` with eta = 1/sqrt(2)): the projection is repeated
    while it shrank ||w|| below eta times its previous value, at most three passes."""
    if len(V) == 0:
        return w, np.zeros(0, dtype=C128)
    B = V.mat()
    nw0 = np.vdot(w, w).real
    h = np.conj(np.conj(w) @ B)
    w = w - B @ h
    nw1 = np.vdot(w, w).real
    passes = 1
    while passes < 3 and nw1 < 0.5 * nw0:
        nw0 = nw1
        h2 = np.conj(np.conj(w) @ B)
        w = w - B @ h2
        h = h + h2
        nw1 = np.vdot(w, w).real
        passes += 1
    return w, h


def _phase_align(v: np.ndarray, x0: np.ndarray) -> np.ndarray:
    """Fix the eigenvector phase so that ``<x0, v>`` is real and non-negative."""
    ov = np.vdot(x0, v)
    if abs(ov) > 0:
        v = v * (np.conj(ov) / abs(ov))
    return v


def lanczos_eigsolve(A: Callable, x0: np.ndarray, tol: float, krylovdim: int = 30,
                     maxiter: int = 300, eager: bool = True, which: str = "SR"):
    """Smallest-real eigenpair of a Hermitian map (``fixedpoint(.., :SR, Lanczos)``,
    ``src/utility.jl:180-186``, ``_eigsolve`` ``:379-393``).

    Thick-restart Lanczos with full CGS2 re-orthogonalisation.  The projected
    matrix is the Hermitian part of the Gram-Schmidt coefficients; a Ritz pair
    is converged when ``|beta_m u_m| <= tol``.  At a restart the
    ``keep = (3 krylovdim + 2 converged) // 5`` best Ritz vectors are kept
    (KrylovKit's shrink rule).  ``maxiter`` counts restart cycles.  The
    returned vector is normalised and phase-aligned with ``x0``.
    """
    shape = x0.shape
    x0f = np.asarray(x0, dtype=C128).ravel(order="F")
    n = x0f.size
    kdim = min(krylovdim, n)
    beta0 = np.linalg.norm(x0f)
    if beta0 == 0:
        raise ValueError("eigsolve: zero starting vector")
    x0n = x0f / beta0
    V = _KBasis(n, kdim + 1, x0n)
    H = np.zeros((kdim + 1, kdim), dtype=C128)
    info = KrylovInfo(numiter=1)
    sign = 1.0 if which == "SR" else -1.0
    while True:
        k = len(V) - 1  # index of the vector to expand
        w = A(freshape(V[k], shape)).ravel(order="F").astype(C128, copy=False)
        info.numops += 1
        w, h = _cgs2(V, w)
        beta = np.linalg.norm(w)
        H[: k + 1, k] = h
        H[k + 1, k] = beta
        m = k + 1
        Hs = H[:m, :m]
        Hs = 0.5 * (Hs + Hs.conj().T)
        theta, U = np.linalg.eigh(Hs)
        order = np.argsort(sign * theta, kind="stable")
        theta, U = theta[order], U[:, order]
        res = np.abs(beta * U[m - 1, :])
        breakdown = beta <= 1e-14 * max(1.0, abs(theta).max())
        full = m == kdim
        if eager or full or breakdown:
            if res[0] <= tol or breakdown:
                info.converged = 1
                info.normres = float(res[0])
                vec = V.mat() @ U[:, 0]
                vec /= np.linalg.norm(vec)
                vec = _phase_align(vec, x0n)
                return float(theta[0]), freshape(vec, shape), info
        if full:
            if info.numiter >= maxiter:
                info.normres = float(res[0])
                vec = V.mat() @ U[:, 0]
                vec /= np.linalg.norm(vec)
                return float(theta[0]), freshape(vec, shape), info
            nconv = int(np.sum(res <= tol))
            keep = max(1, (3 * kdim + 2 * nconv) // 5)
            Vk = V.mat() @ U[:, :keep]
            V.reset(Vk)
            V.append(w / beta)
            H = np.zeros((kdim + 1, kdim), dtype=C128)
            H[:keep, :keep] = np.diag(theta[:keep])
            H[keep, :keep] = beta * U[m - 1, :keep]
            info.numiter += 1
        else:
            V.append(w / beta)


def gmres(A: Callable, b: np.ndarray, x0: np.ndarray, tol: float, krylovdim: int = 30,
          maxiter: int = 300, a0: complex = 1.0, a1: complex = 1.0):
    """``linsolve(op, b, x0, GMRES; a0, a1)`` solving ``(a0 + a1 A) x = b``
    (``src/algorithms/groundstates/envs.jl:14-19``).

    Restarted GMRES(krylovdim) with CGS2 and Givens rotations; ``tol`` bounds
    the 2-norm of the residual; ``maxiter`` counts restart cycles.  The true
    residual is recomputed after every cycle.
    """
    shape = b.shape
    bf = np.asarray(b, dtype=C128).ravel(order="F")
    x = np.asarray(x0, dtype=C128).ravel(order="F").copy()
    info = KrylovInfo()

    def op(v):
        info.numops += 1
        return a0 * v + a1 * A(freshape(v, shape)).ravel(order="F")

    r = bf - op(x)
    beta = np.linalg.norm(r)
    info.normres = float(beta)
    if beta <= tol:
        info.converged = 1
        return freshape(x, shape), info
    n = bf.size
    kdim = min(krylovdim, n)
    while True:
        info.numiter += 1
        V = _KBasis(n, kdim + 1, r / beta)
        R = np.zeros((kdim + 1, kdim), dtype=C128)
        cs = np.zeros(kdim, dtype=np.float64)
        sn = np.zeros(kdim, dtype=C128)
        g = np.zeros(kdim + 1, dtype=C128)
        g[0] = beta
        kused = 0
        for k in range(kdim):
            w = op(V[k])
            w, h = _cgs2(V, w)
            hn = np.linalg.norm(w)
            col = np.zeros(k + 2, dtype=C128)
            col[: k + 1] = h
            col[k + 1] = hn
            for j in range(k):
                t1 = cs[j] * col[j] + sn[j] * col[j + 1]
                col[j + 1] = -np.conj(sn[j]) * col[j] + cs[j] * col[j + 1]
                col[j] = t1
            a, bb = col[k], col[k + 1]
            nrm = math.hypot(abs(a), abs(bb))
            if nrm == 0:
                cs[k], sn[k] = 1.0, 0.0
            elif abs(a) == 0:
                cs[k], sn[k] = 0.0, np.conj(bb) / abs(bb)
                cs[k] = 0.0
            else:
                cs[k] = abs(a) / nrm
                sn[k] = (a / abs(a)) * np.conj(bb) / nrm
            col[k] = cs[k] * a + sn[k] * bb
            col[k + 1] = 0.0
            g[k + 1] = -np.conj(sn[k]) * g[k]
            g[k] = cs[k] * g[k]
            R[: k + 2, k] = col
            kused = k + 1
            if abs(g[k + 1]) <= tol or hn <= 1e-300:
                break
            V.append(w / hn)
        # back substitution
        y = np.zeros(kused, dtype=C128)
        for i in range(kused - 1, -1, -1):
            y[i] = (g[i] - R[i, i + 1:kused] @ y[i + 1:kused]) / R[i, i]
        x = x + V.mat(kused) @ y
        r = bf - op(x)
        beta = np.linalg.norm(r)
        info.normres = float(beta)
        if beta <= tol:
            info.converged = 1
            return freshape(x, shape), info
        if info.numiter >= maxiter:
            return freshape(x, shape), info


def _expm_herm(Hs: np.ndarray, t: complex) -> np.ndarray:
    th, U = np.linalg.eigh(Hs)
    return (U * np.exp(t * th)[None, :]) @ U.conj().T


def exponentiate(A: Callable, t: complex, x: np.ndarray, tol: float = 1e-10,
                 krylovdim: int = 30, maxiter: int = 300):
    """``exponentiate(A, t, x; ishermitian = true)`` (``src/algorithms/timeevo/tdvp.jl:14-20``).

    Lanczos (full CGS2) Krylov exponential with time sub-stepping.  For a
    remaining step ``tau`` the a-posteriori error estimate of the basis of size
    ``m`` is ``beta |h_{m+1,m}| |[exp(tau H_m) e1]_m|``; a step is accepted when
    the estimate is at most ``tol |tau| / |t|``.  When the basis is full and the
    whole remainder is not accepted, ``tau`` is halved until it is.  ``maxiter``
    bounds the number of accepted sub-steps.
    """
    shape = x.shape
    v = np.asarray(x, dtype=C128).ravel(order="F").copy()
    info = KrylovInfo()
    T = complex(t)
    if T == 0:
        info.converged = 1
        return freshape(v, shape), info
    remaining = T
    n = v.size
    kdim = min(krylovdim, n)
    while True:
        beta = np.linalg.norm(v)
        if beta == 0:
            info.converged = 1
            return freshape(v, shape), info
        info.numiter += 1
        V = _KBasis(n, kdim + 1, v / beta)
        H = np.zeros((kdim + 1, kdim), dtype=C128)
        tau = remaining
        accepted = False
        while True:
            k = len(V) - 1
            w = A(freshape(V[k], shape)).ravel(order="F").astype(C128, copy=False)
            info.numops += 1
            w, h = _cgs2(V, w)
            hn = np.linalg.norm(w)
            H[: k + 1, k] = h
            H[k + 1, k] = hn
            m = k + 1
            Hs = H[:m, :m]
            Hs = 0.5 * (Hs + Hs.conj().T)
            breakdown = hn <= 1e-14 * max(1.0, np.abs(np.diag(Hs)).max())
            E = _expm_herm(Hs, tau)
            err = beta * hn * abs(E[m - 1, 0])
            if breakdown or err <= tol * abs(tau) / abs(T):
                accepted = True
                break
            if m == kdim:
                while err > tol * abs(tau) / abs(T) and abs(tau) > 1e-300:
                    tau = tau / 2
                    E = _expm_herm(Hs, tau)
                    err = beta * hn * abs(E[m - 1, 0])
                accepted = True
                break
            V.append(w / hn)
        if accepted:
            m = len(V)
            E = _expm_herm(Hs, tau)
            v = beta * (V.mat() @ E[:, 0])
            remaining = remaining - tau
            info.normres = float(err)
            if abs(remaining) <= 1e-15 * abs(T):
                info.converged = 1
                return freshape(v, shape), info
            if info.numiter >= maxiter:
                return freshape(v, shape), info


def _schur_sorted(M: np.ndarray):
    """Complex Schur form ``M = Z T Z^H`` with ``|T[k,k]|`` non-increasing.

    LAPACK's Schur form (scipy) reordered by adjacent swaps: the block
    ``[[t11, t12], [0, t22]]`` has the eigenvector ``(t12, t22 - t11)`` for ``t22``,
    and the unitary built from it moves ``t22`` up (LAPACK ``ztrexc``'s step)."""
    import scipy.linalg as sl
    T, Z = sl.schur(np.asarray(M, dtype=C128), output="complex")
    T = np.array(T, dtype=C128)
    Z = np.array(Z, dtype=C128)
    n = T.shape[0]
    for _ in range(n):
        swapped = False
        for k in range(n - 1):
            t11, t22 = T[k, k], T[k + 1, k + 1]
            if not abs(t22) > abs(t11):
                continue
            g = np.array([T[k, k + 1], t22 - t11])
            nr = np.linalg.norm(g)
            if nr == 0.0:
                continue
            g /= nr
            G = np.array([[g[0], -np.conj(g[1])], [g[1], np.conj(g[0])]])
            T[k:k + 2, :] = G.conj().T @ T[k:k + 2, :]
            T[:, k:k + 2] = T[:, k:k + 2] @ G
            Z[:, k:k + 2] = Z[:, k:k + 2] @ G
            T[k + 1, k] = 0.0
            T[k, k], T[k + 1, k + 1] = t22, t11
            swapped = True
        if not swapped:
            break
    return T, Z


def arnoldi_dominant(A: Callable, x0: np.ndarray, tol: float, krylovdim: int = 30,
                     maxiter: int = 300, eager: bool = True):
    """Dominant (largest-magnitude) eigenpair of a non-Hermitian map.

    Restates ``gauge_fixedpoint`` (KrylovKit ``schursolve``, ``src/utility.jl:204-211``)
    and the ``:LM`` Arnoldi of ``dot(psi, psi)`` (``src/states/canonicalmps.jl:262-269``).
    Arnoldi with CGS2 in Krylov-Schur form ``A V_m = V_{m+1} H``; a Ritz pair ``(lam, V y)``
    is converged when ``|H[m, :] y| <= tol`` (``y`` normalised).  A full basis restarts
    from the leading ``keep = (3 krylovdim + 2 nconv) // 5`` Schur vectors of ``H[:m, :m]``
    (sorted by ``|lambda|``) plus the residual vector, as ``schursolve`` does.  The vector
    is normalised and phase-aligned with ``x0``.
    """
    shape = x0.shape
    x0f = np.asarray(x0, dtype=C128).ravel(order="F")
    n = x0f.size
    kdim = min(krylovdim, n)
    x0n = x0f / np.linalg.norm(x0f)
    V = _KBasis(n, kdim + 1, x0n)
    H = np.zeros((kdim + 1, kdim), dtype=C128)
    info = KrylovInfo(numiter=1)
    while True:
        k = len(V) - 1
        w = A(freshape(V[k], shape)).ravel(order="F").astype(C128, copy=False)
        info.numops += 1
        w, h = _cgs2(V, w)
        hn = np.linalg.norm(w)
        H[: k + 1, k] = h
        H[k + 1, k] = hn
        m = k + 1
        lam, Y = np.linalg.eig(H[:m, :m])
        j = int(np.argmax(np.abs(lam)))
        y = Y[:, j] / np.linalg.norm(Y[:, j])
        res = abs(H[m, :m] @ y)
        breakdown = hn <= 1e-14 * max(1.0, abs(lam[j]))
        full = m == kdim
        if eager or full or breakdown:
            if res <= tol or breakdown:
                info.converged = 1
                info.normres = float(res)
                vec = V.mat() @ y
                vec /= np.linalg.norm(vec)
                return complex(lam[j]), freshape(_phase_align(vec, x0n), shape), info
        if full:
            if info.numiter >= maxiter:
                vec = V.mat() @ y
                vec /= np.linalg.norm(vec)
                info.normres = float(res)
                return complex(lam[j]), freshape(vec, shape), info
            T, Z = _schur_sorted(H[:m, :m])
            nconv = 1 if res <= tol else 0
            keep = max(1, min(m - 1, (3 * kdim + 2 * nconv) // 5))
            Vm = V.mat() @ Z[:, :keep]
            Hn = np.zeros((kdim + 1, kdim), dtype=C128)
            Hn[:keep, :keep] = np.triu(T[:keep, :keep])
            Hn[keep, :keep] = H[m, :m] @ Z[:, :keep]
            V.reset(Vm)
            V.append(w / hn)
            H = Hn
            info.numiter += 1
        else:
            V.append(w / hn)


# --------------------------------------------------------------------------
# Transfer pushes  (src/transfermatrix.jl:5-66, src/algorithms/groundstates/envs.jl:104-114, 199-231)
# --------------------------------------------------------------------------
def push_env_left(L, above, below=None):
    """``L'[a',b'] = sum conj(below[a,s,a']) L[a,b] above[b,s,b']`` (``transfermatrix.jl:5-7, 54-58``)."""
    below = above if below is None else below
    Dl, d, Dr = above.shape
    Y = L @ freshape(above, (Dl, d * Dr))
    return np.asfortranarray(freshape(below, (below.shape[0] * d, below.shape[2])).conj().T @ freshape(Y, (Dl * d, Dr)))


def push_env_right(R, above, below=None):
    """``R'[a',b'] = sum above[a',s,a] R[a,b] conj(below[b',s,b])`` (``transfermatrix.jl:23-26, 62-66``)."""
    below = above if below is None else below
    Dl, d, Dr = above.shape
    Y = freshape(above, (Dl * d, Dr)) @ R
    return np.asfortranarray(freshape(Y, (Dl, d * R.shape[1])) @ freshape(below, (below.shape[0], d * below.shape[2])).conj().T)


def push_slice_left(L, Wl, A):
    """``_push_slice_left`` (``envs.jl:104-107``): ``sum conj(A[a,u,a']) L[a,b] Wl[u,d] A[b,d,b']``."""
    Dl, d, Dr = A.shape
    Y = freshape(L @ freshape(A, (Dl, d * Dr)), (Dl, d, Dr))
    Z = np.einsum("ud,adb->aub", Wl, Y, optimize=True)
    return np.asfortranarray(freshape(A, (Dl * d, Dr)).conj().T @ freshape(np.asfortranarray(Z), (Dl * d, Dr)))


def push_slice_right(R, Wl, A):
    """``_push_slice_right`` (``envs.jl:111-114``): ``sum A[a',d,a] R[a,b] Wl[u,d] conj(A[b',u,b])``."""
    Dl, d, Dr = A.shape
    Y = freshape(freshape(A, (Dl * d, Dr)) @ R, (Dl, d, Dr))
    Z = np.einsum("ud,adb->aub", Wl, Y, optimize=True)
    return np.asfortranarray(freshape(np.asfortranarray(Z), (Dl, d * Dr)) @ freshape(A, (Dl, d * Dr)).conj().T)


def push_mpo_left(L, W, A):
    """Schur/dense MPO left push (``envs.jl:199-210``, ``transfermatrix.jl:11-13``):
    ``L'[a',j,b'] = sum conj(A[a,u,a']) L[a,i,b] W[i,u,j,d] A[b,d,b']``."""
    Dl, d, Dr = A.shape
    m, n = W.shape[0], W.shape[2]
    Y = freshape(freshape(L, (Dl * m, Dl)) @ freshape(A, (Dl, d * Dr)), (Dl, m, d, Dr))
    Z = np.einsum("iujd,aidb->aujb", W, Y, optimize=True)
    out = freshape(A, (Dl * d, Dr)).conj().T @ freshape(np.asfortranarray(Z), (Dl * d, n * Dr))
    return np.asfortranarray(freshape(out, (Dr, n, Dr)))


def push_mpo_right(R, W, A):
    """Schur/dense MPO right push (``envs.jl:220-231``, ``transfermatrix.jl:31-35``):
    ``R'[a',i,b'] = sum A[a',d,a] W[i,u,j,d] conj(A[b',u,b]) R[a,j,b]``."""
    Dl, d, Dr = A.shape
    m, n = W.shape[0], W.shape[2]
    Y = freshape(freshape(A, (Dl * d, Dr)) @ freshape(R, (Dr, n * Dr)), (Dl, d, n, Dr))
    Z = np.einsum("iujd,adjb->aiub", W, Y, optimize=True)
    out = freshape(np.asfortranarray(Z), (Dl * m, d * Dr)) @ freshape(A, (Dl, d * Dr)).conj().T
    return np.asfortranarray(freshape(out, (Dl, m, Dl)))


def regularize(v, lvec, rvec):
    """``regularize!(v, lvec, rvec)`` (``envs.jl:28-32``): ``v - tr(lvec v) rvec`` (no conjugation)."""
    c = np.sum(lvec * v.T)
    return np.asfortranarray(v - c * rvec)


# --------------------------------------------------------------------------
# States: CanonicalIMPS and gauge fixing  (src/states/canonicalmps.jl, ortho.jl)
# --------------------------------------------------------------------------
@dataclass
class CanonicalIMPS:
    """``CanonicalIMPS`` (``canonicalmps.jl:17-40``): ``AL[i] C[i] = AC[i] = C[i-1] AR[i]``."""
    AL: List[np.ndarray]
    AR: List[np.ndarray]
    C: List[np.ndarray]
    AC: List[np.ndarray]

    def __len__(self):
        return len(self.AL)

    def copy(self):
        return CanonicalIMPS([a.copy(order="F") for a in self.AL], [a.copy(order="F") for a in self.AR],
                             [c.copy(order="F") for c in self.C], [a.copy(order="F") for a in self.AC])

    def Cm(self, l):
        """Periodic access to ``C[l]`` with Julia's 1-based site labels (``C[0] = C[N]``)."""
        return self.C[(l - 1) % len(self.C)]


def _mulAL(AL, C):
    Dl, d, Dr = AL.shape
    return np.asfortranarray(freshape(freshape(AL, (Dl * d, Dr)) @ C, (Dl, d, C.shape[1])))


def _mulCA(C, A):
    Dl, d, Dr = A.shape
    return np.asfortranarray(freshape(C @ freshape(A, (Dl, d * Dr)), (C.shape[0], d, Dr)))


def _fnorm(x):
    return float(np.linalg.norm(np.asarray(x).ravel()))


def _gauge_eig_tol(eps):
    # _GAUGE_ALG_EIGSOLVE = alg_eigsolve(ishermitian=false, tol_factor=1)  (ortho.jl:6)
    return min(max(eps ** 2, Defaults.tol_min), Defaults.tol_max)


def uniform_leftorth(A: List[np.ndarray], C0: np.ndarray, tol=Defaults.tolgauge,
                     maxiter=Defaults.maxiter, eig_miniter=10):
    """``uniform_leftorth!`` (``ortho.jl:125-164``). Returns ``(AL, C, info)``,
    ``C[i]`` the bond matrix right of site ``i`` (0-based list, ``C[-1] = C[N]``)."""
    N = len(A)
    Awork = [a.copy(order="F") for a in A]
    C = [None] * N
    C[N - 1] = C0 / _fnorm(C0)
    AL = [None] * N
    it = 0
    eps = math.inf
    while True:
        if it >= eig_miniter:
            etol = _gauge_eig_tol(eps)

            def tm(v):
                L = v
                for l in range(N):
                    L = push_env_left(L, Awork[l], AL[l])
                return L
            _, evec, _ = arnoldi_dominant(tm, C[N - 1], etol)
            _, C[N - 1] = qrpos(evec)
        Cpre = C[N - 1].copy()
        for i in range(N):
            Dl_, d, Dr_ = Awork[i].shape
            M = _mulCA(C[i - 1], Awork[i])
            Q, Rf = qrpos(freshape(M, (M.shape[0] * d, Dr_)))
            AL[i] = np.asfortranarray(freshape(Q, (M.shape[0], d, Q.shape[1])))
            C[i] = Rf
        C[N - 1] = C[N - 1] / _fnorm(C[N - 1])
        eps = _fnorm(C[N - 1] - Cpre)
        it += 1
        if eps < tol or it > maxiter:
            return AL, C, dict(niter=it, err=eps, converged=eps < tol)


def uniform_rightorth(A: List[np.ndarray], C0: np.ndarray, tol=Defaults.tolgauge,
                      maxiter=Defaults.maxiter, eig_miniter=10):
    """``uniform_rightorth!`` (``ortho.jl:166-202``). Returns ``(AR, C, info)``."""
    N = len(A)
    Awork = [a.copy(order="F") for a in A]
    C = [None] * N
    C[N - 1] = C0 / _fnorm(C0)
    AR = [None] * N
    it = 0
    eps = math.inf
    while True:
        if it >= eig_miniter:
            etol = _gauge_eig_tol(eps)

            def tm(v):
                R = v
                for l in range(N - 1, -1, -1):
                    R = push_env_right(R, Awork[l], AR[l])
                return R
            _, evec, _ = arnoldi_dominant(tm, C[N - 1], etol)
            C[N - 1], _ = lqpos(evec)
        Cpre = C[N - 1].copy()
        for i in range(N - 1, -1, -1):
            Dl_, d, Dr_ = Awork[i].shape
            M = _mulAL(Awork[i], C[i])
            Lf, Q = lqpos(freshape(M, (Dl_, d * M.shape[2])))
            AR[i] = np.asfortranarray(freshape(Q, (Lf.shape[1], d, M.shape[2])))
            C[i - 1] = Lf
        C[N - 1] = C[N - 1] / _fnorm(C[N - 1])
        eps = _fnorm(C[N - 1] - Cpre)
        it += 1
        if eps < tol or it > maxiter:
            return AR, C, dict(niter=it, err=eps, converged=eps < tol)


def gaugefix(A: List[np.ndarray], C0: np.ndarray, order="LR", tol=Defaults.tolgauge,
             maxiter=Defaults.maxiter, AL_given=None) -> CanonicalIMPS:
    """``gaugefix!`` (``ortho.jl:64-99``) returning a fresh ``CanonicalIMPS``.

    ``order='LR'``: left-orthogonalise ``A`` from ``C0``, then right-orthogonalise
    the resulting ``AL`` from ``C[N]``; ``AC = AL C``.  ``order='R'``: ``AL`` is
    kept as given (``A``), ``AR, C`` come from ``uniform_rightorth!``; ``AC = C AR``.
    """
    N = len(A)
    if order == "LR":
        AL, C, _ = uniform_leftorth(A, C0, tol, maxiter)
        AR, C, _ = uniform_rightorth(AL, C[N - 1], tol, maxiter)
        AC = [_mulCA(C[i - 1], AR[i]) for i in range(N)]
        return CanonicalIMPS(AL, AR, C, AC)
    if order == "R":
        AL = [a.copy(order="F") for a in A]
        AR, C, _ = uniform_rightorth(A, C0, tol, maxiter)
        AC = [_mulCA(C[i - 1], AR[i]) for i in range(N)]
        return CanonicalIMPS(AL, AR, C, AC)
    raise ValueError(f"invalid order {order}")


def canonical_from_AL(ALs: List[np.ndarray], C0: np.ndarray, tol=Defaults.tolgauge,
                      maxiter=Defaults.maxiter) -> CanonicalIMPS:
    """``CanonicalIMPS(ALs, C0)`` (``canonicalmps.jl:180-195``): right gauge fix, ``AC = AL C``."""
    psi = gaugefix(ALs, C0, order="R", tol=tol, maxiter=maxiter)
    psi.AC = [_mulAL(psi.AL[i], psi.C[i]) for i in range(len(ALs))]
    return psi


def canonical_from_sites(As: List[np.ndarray], tol=Defaults.tolgauge, maxiter=Defaults.maxiter):
    """``CanonicalIMPS(As)`` (``canonicalmps.jl:151-170``) for full-rank uniform-bond input:
    ``gaugefix!(:LR)`` from ``C0 = I`` then ``AC = AL C``."""
    D = As[0].shape[0]
    psi = gaugefix(As, np.eye(D, dtype=C128, order="F"), order="LR", tol=tol, maxiter=maxiter)
    psi.AC = [_mulAL(psi.AL[i], psi.C[i]) for i in range(len(As))]
    return psi


def random_site_tensors(dims: Sequence[int], D: int, seed: int) -> List[np.ndarray]:
    """Seeded i.i.d. complex-normal site tensors (Re, Im ~ N(0, 1/2)), NumPy PCG64.

    Stands in for Julia's ``randn(rng, ComplexF64, D, d, D)`` (``constructors.jl:13-22``);
    the same arrays are fed to the oracle and to the GPU.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for d in dims:
        re = rng.standard_normal((D, d, D))
        im = rng.standard_normal((D, d, D))
        out.append(np.asfortranarray((re + 1j * im) / math.sqrt(2.0)))
    return out


def randomimps(dims: Sequence[int], D: int, seed: int, **kw) -> CanonicalIMPS:
    """``randomimps(ComplexF64, dims; D)`` (``constructors.jl:13-22``) with a PCG64 seed."""
    return canonical_from_sites(random_site_tensors(dims, D, seed), **kw)


def regauge(AC: np.ndarray, C: np.ndarray) -> np.ndarray:
    """``regauge!(AC, C)`` (``ortho.jl:214-219``): ``AL = Q(AC) Q(C)^H`` with QRpos."""
    Dl, d, Dr = AC.shape
    Qac, _ = qrpos(freshape(AC, (Dl * d, Dr)))
    Qc, _ = qrpos(C)
    return np.asfortranarray(freshape(Qac @ Qc.conj().T, (Dl, d, Dr)))


def state_dot(psi1: CanonicalIMPS, psi2: CanonicalIMPS, krylovdim=Defaults.krylovdim) -> complex:
    """``dot(psi1, psi2)`` (``canonicalmps.jl:262-269``): dominant eigenvalue of
    ``TransferMatrix(psi2.AL, psi1.AL)`` from ``v0 = I`` (Arnoldi, ``tol = 1e-10``)."""
    N = len(psi1)
    D0 = psi1.AL[0].shape[0]
    v0 = np.eye(D0, psi2.AL[0].shape[0], dtype=C128, order="F")

    def tm(v):
        L = v
        for l in range(N):
            L = push_env_left(L, psi2.AL[l], psi1.AL[l])
        return L
    lam, _, _ = arnoldi_dominant(tm, v0, Defaults.tol, krylovdim)
    return lam


# --------------------------------------------------------------------------
# Environments: DMRGCache(psi, ::SparseIMPO)  (src/algorithms/groundstates/envs.jl:121-188, 321-546)
# --------------------------------------------------------------------------
@dataclass
class DMRGCache:
    """Schur-Hamiltonian environments: ``lefts[l]`` is ``(chi_{l-1}, m_l, chi_{l-1})``
    (bra, level, ket) and ``rights[l]`` is ``(chi_l, n_l, chi_l)`` (ket, level, bra)."""
    lefts: List[np.ndarray]
    rights: List[np.ndarray]
    stats: dict = field(default_factory=dict)

    def leftenv(self, l):
        return self.lefts[l % len(self.lefts)]

    def rightenv(self, l):
        return self.rights[l % len(self.rights)]


def _left_cyclethrough(lefts, H, AL, i, N):
    """``_left_cyclethrough!`` (``envs.jl:121-136``); ``i`` is 1-based; zero blocks skipped."""
    for site in range(N):
        snext = (site + 1) % N
        chi = AL[site].shape[2]
        W = H[site]
        ms, ns = W.shape[0], W.shape[2]
        if not (i <= ns - 1):
            continue
        tgt = fzeros((chi, chi))
        for l in range(1, min(i, ms) + 1):
            blk = W[l - 1, :, i - 1, :]
            if not np.any(blk):
                continue
            tgt += push_slice_left(np.asfortranarray(lefts[site][:, l - 1, :]), blk, AL[site])
        lefts[snext][:, i - 1, :] = tgt


def _left_closing_sweep(lefts, H, AL, N):
    """``_left_closing_sweep!`` (``envs.jl:143-156``)."""
    for site in range(N):
        snext = (site + 1) % N
        chi = AL[site].shape[2]
        W = H[site]
        ms, ns = W.shape[0], W.shape[2]
        tgt = fzeros((chi, chi))
        for l in range(1, ms + 1):
            blk = W[l - 1, :, ns - 1, :]
            if not np.any(blk):
                continue
            tgt += push_slice_left(np.asfortranarray(lefts[site][:, l - 1, :]), blk, AL[site])
        lefts[snext][:, ns - 1, :] = tgt


def _right_cyclethrough(rights, H, AR, i, N):
    """``_right_cyclethrough!`` (``envs.jl:162-177``)."""
    for site in range(N - 1, -1, -1):
        sprev = (site - 1) % N
        chi = AR[site].shape[0]
        W = H[site]
        ms, ns = W.shape[0], W.shape[2]
        if not (i <= ms):
            continue
        tgt = fzeros((chi, chi))
        for l in range(i, ns + 1):
            blk = W[i - 1, :, l - 1, :]
            if not np.any(blk):
                continue
            tgt += push_slice_right(np.asfortranarray(rights[site][:, l - 1, :]), blk, AR[site])
        rights[sprev][:, i - 1, :] = tgt


def _diag_channel(W, i):
    """``_diag_channel`` (``envs.jl:182-188``)."""
    if i <= min(W.shape[0], W.shape[2]):
        return W[i - 1, :, i - 1, :]
    return np.zeros((W.shape[1], W.shape[3]), dtype=C128)


def build_envs(psi: CanonicalIMPS, H: SchurMPO, tol=Defaults.tol, maxiter=Defaults.maxiter,
               krylovdim=Defaults.krylovdim, init: Optional[DMRGCache] = None) -> DMRGCache:
    """``DMRGCache(psi, H::SparseIMPO; tol, maxiter, krylovdim, init_lefts, init_rights)``
    (``envs.jl:321-518``), step for step."""
    N = len(psi)
    Dl = [psi.AL[l].shape[0] for l in range(N)]
    Dr = [psi.AL[l].shape[2] for l in range(N)]
    if H[N - 1].shape[2] != H[0].shape[0]:
        raise ValueError("operator level chain does not close over the ket unit cell")
    ml = [H[l].shape[0] for l in range(N)]
    nr = [H[l].shape[2] for l in range(N)]
    lefts = [fzeros((Dl[l], ml[l], Dl[l])) for l in range(N)]
    rights = [fzeros((Dr[l], nr[l], Dr[l])) for l in range(N)]
    for l in range(N):
        lefts[l][:, 0, :] = np.eye(Dl[l])
        rights[l][:, nr[l] - 1, :] = np.eye(Dr[l])
    kdim = min(Dl[0] * Dl[0], krylovdim)
    stats = dict(gmres_iters=0, gmres_ops=0, solves=0)
    AL, AR = psi.AL, psi.AR

    def solve(op, rhs, prev):
        x, info = gmres(op, rhs, prev, tol, kdim, maxiter, 1.0, -1.0)
        stats["gmres_iters"] += info.numiter
        stats["gmres_ops"] += info.numops
        stats["solves"] += 1
        return x

    CN = psi.C[N - 1]
    jmax = max(nr) - 1
    # ---- left environments (envs.jl:363-421)
    for i in range(2, jmax + 1):
        if i <= ml[0] - 1:
            D = Dl[0]
            if init is not None and init.lefts[0].shape == lefts[0].shape:
                prev = np.asfortranarray(init.lefts[0][:, i - 1, :])
            else:
                prev = np.asfortranarray(lefts[0][:, i - 1, :])
            _left_cyclethrough(lefts, H, AL, i, N)
            rhs = np.asfortranarray(lefts[0][:, i - 1, :])
            if H.isidentitylevel(i):
                rho_r = CN @ CN.conj().T
                I1 = np.eye(D, dtype=C128)

                def op(v):
                    X = v
                    for l in range(N):
                        X = push_env_left(X, AL[l])
                    return regularize(X, rho_r, I1)
                lefts[0][:, i - 1, :] = solve(op, rhs, prev)
                if N > 1:
                    _left_cyclethrough(lefts, H, AL, i, N)
                for l in range(N):
                    Cp = psi.C[l - 1]
                    lefts[l][:, i - 1, :] = regularize(np.asfortranarray(lefts[l][:, i - 1, :]), Cp @ Cp.conj().T, np.eye(Dl[l]))
            else:
                if not H.isemptylevel(i):
                    def op(v, i=i):
                        X = v
                        for l in range(N):
                            blk = _diag_channel(H[l], i)
                            X = push_slice_left(X, blk, AL[l]) if np.any(blk) else fzeros((AL[l].shape[2], AL[l].shape[2]))
                        return X
                    lefts[0][:, i - 1, :] = solve(op, rhs, prev)
                if N > 1:
                    _left_cyclethrough(lefts, H, AL, i, N)
        else:
            _left_cyclethrough(lefts, H, AL, i, N)
    # ---- closing level of the left environments (envs.jl:424-455)
    i = ml[0]
    D = Dl[0]
    if init is not None and init.lefts[0].shape == lefts[0].shape:
        prev = np.asfortranarray(init.lefts[0][:, i - 1, :])
    else:
        prev = np.asfortranarray(lefts[0][:, i - 1, :])
    _left_closing_sweep(lefts, H, AL, N)
    rhs = np.asfortranarray(lefts[0][:, i - 1, :])
    rho_r = CN @ CN.conj().T
    I1 = np.eye(D, dtype=C128)

    def opL(v):
        X = v
        for l in range(N):
            X = push_env_left(X, AL[l])
        return regularize(X, rho_r, I1)
    lefts[0][:, i - 1, :] = solve(opL, rhs, prev)
    if N > 1:
        _left_closing_sweep(lefts, H, AL, N)
    for l in range(N):
        Cp = psi.C[l - 1]
        lefts[l][:, ml[l] - 1, :] = regularize(np.asfortranarray(lefts[l][:, ml[l] - 1, :]), Cp @ Cp.conj().T, np.eye(Dl[l]))
    # ---- right environments (envs.jl:461-515)
    for i in range(jmax, 0, -1):
        if i <= nr[N - 1] - 1:
            D = Dr[N - 1]
            if init is not None and init.rights[N - 1].shape == rights[N - 1].shape:
                prev = np.asfortranarray(init.rights[N - 1][:, i - 1, :])
            else:
                prev = np.asfortranarray(rights[N - 1][:, i - 1, :])
            _right_cyclethrough(rights, H, AR, i, N)
            rhs = np.asfortranarray(rights[N - 1][:, i - 1, :])
            if H.isidentitylevel(i):
                rho_l = CN.conj().T @ CN
                IN = np.eye(D, dtype=C128)

                def op(v):
                    X = v
                    for l in range(N - 1, -1, -1):
                        X = push_env_right(X, AR[l])
                    return regularize(X, rho_l, IN)
                rights[N - 1][:, i - 1, :] = solve(op, rhs, prev)
                if N > 1:
                    _right_cyclethrough(rights, H, AR, i, N)
                for l in range(N):
                    Cl = psi.C[l]
                    rights[l][:, i - 1, :] = regularize(np.asfortranarray(rights[l][:, i - 1, :]), Cl.conj().T @ Cl, np.eye(Dr[l]))
            else:
                if not H.isemptylevel(i):
                    def op(v, i=i):
                        X = v
                        for l in range(N - 1, -1, -1):
                            blk = _diag_channel(H[l], i)
                            X = push_slice_right(X, blk, AR[l]) if np.any(blk) else fzeros((AR[l].shape[0], AR[l].shape[0]))
                        return X
                    rights[N - 1][:, i - 1, :] = solve(op, rhs, prev)
                if N > 1:
                    _right_cyclethrough(rights, H, AR, i, N)
        else:
            _right_cyclethrough(rights, H, AR, i, N)
    return DMRGCache(lefts, rights, stats)


# --------------------------------------------------------------------------
# Effective Hamiltonians  (src/algorithms/groundstates/effective.jl:72-102)
# --------------------------------------------------------------------------
def ac_apply(GL, W, GR, x):
    """``MPO_AC_Hamiltonian`` action (``effective.jl:79-102``):
    ``y[b,u,c] = sum GL[b,i,a] x[a,s,bb] W[i,u,j,s] GR[bb,j,c]`` (linear, no conj).

    Contraction order: ``GL x`` (one GEMM over all left levels), the W mixing,
    then one GEMM with ``GR`` over all right levels.
    """
    Dl, d, Dr = x.shape
    m, n = W.shape[0], W.shape[2]
    T1 = freshape(freshape(GL, (Dl * m, Dl)) @ freshape(x, (Dl, d * Dr)), (Dl, m, d, Dr))
    T2 = np.asfortranarray(np.einsum("iujs,bisc->bucj", W, T1, optimize=True))
    y = freshape(T2, (Dl * d, Dr * n)) @ freshape(GR, (Dr * n, GR.shape[2]))
    return np.asfortranarray(freshape(y, (Dl, d, GR.shape[2])))


def c_apply(GL, GR, x):
    """``MPO_C_Hamiltonian`` action (``effective.jl:72-76``):
    ``y[a,b] = sum GL[a,w,a'] x[a',b'] GR[b',w,b]``."""
    D1, w, _ = GL.shape
    D2 = x.shape[1]
    T = freshape(freshape(GL, (D1 * w, D1)) @ x, (D1, w, D2))
    T = np.asfortranarray(T.transpose(0, 2, 1))  # [a, b', w]
    y = freshape(T, (D1, D2 * w)) @ freshape(GR, (D2 * w, GR.shape[2]))
    return np.asfortranarray(y)


def calc_galerkin(psi: CanonicalIMPS, H: SchurMPO, envs: DMRGCache) -> float:
    """``calc_galerkin`` (``src/algorithms/groundstates/vumps.jl:111-124``)."""
    eps = 0.0
    for site in range(len(psi)):
        x = ac_apply(envs.lefts[site], H[site], envs.rights[site], psi.AC[site])
        x = x / _fnorm(x)
        AL = psi.AL[site]
        Dl, d, Dr = AL.shape
        A2 = freshape(AL, (Dl * d, Dr))
        x2 = freshape(x, (Dl * d, Dr))
        q = A2.conj().T @ x2
        eps = max(eps, _fnorm(x2 - A2 @ q))
    return eps


def expectationvalue(psi: CanonicalIMPS, H: SchurMPO, envs: DMRGCache) -> complex:
    """Schur energy (``src/observables/expval.jl:93-112``): per site the closing column
    ``sum_l <AC| GL_l W[l, n] GR_n |AC>``, divided by ``dot(psi, psi)``."""
    E = 0.0j
    for site in range(len(psi)):
        W = H[site]
        ms, ns = W.shape[0], W.shape[2]
        Wcol = fzeros((ms, W.shape[1], 1, W.shape[3]))
        Wcol[:, :, 0, :] = W[:, :, ns - 1, :]
        GR = envs.rights[site]
        GRe = np.asfortranarray(GR[:, ns - 1:ns, :])
        y = ac_apply(envs.lefts[site], Wcol, GRe, psi.AC[site])
        E += np.vdot(psi.AC[site], y)
    return E / state_dot(psi, psi)


def local_expectation1(psi: CanonicalIMPS, site: int, O: np.ndarray) -> complex:
    """``_local_expectation1`` (``expval.jl:33-37``)."""
    AC = psi.AC[site]
    E = np.einsum("aub,us,asb->", AC.conj(), O, AC)
    return E / state_dot(psi, psi)


# --------------------------------------------------------------------------
# Energy gradients.  No counterpart in the reference: an extension for
# gradient-based optimisation, derived from the energy functional above.  The
# right environments solve the adjoint of the left fixed-point system, so each
# derivative is one contraction with the converged environments.  Pinned by
# central finite differences in the tests (no reference values exist).
# --------------------------------------------------------------------------
def energy_grad_mpo(psi: CanonicalIMPS, H: SchurMPO, envs: DMRGCache) -> List[np.ndarray]:
    """``dE/dW[site][i,u,j,s] = sum conj(AC[b,u,c']) GL[b,i,a] AC[a,s,c] GR[c,j,c']``
    for every site, with the two identity blocks of the Schur form set to zero."""
    out = []
    for l in range(len(psi)):
        AC = psi.AC[l]
        G = np.einsum("buc,bia,asd,djc->iujs", AC.conj(), envs.lefts[l], AC, envs.rights[l], optimize=True)
        G = np.asfortranarray(G)
        m, n = G.shape[0], G.shape[2]
        G[0, :, 0, :] = 0.0
        G[m - 1, :, n - 1, :] = 0.0
        out.append(G)
    return out


def energy_grad_al(psi: CanonicalIMPS, H: SchurMPO, envs: DMRGCache) -> List[np.ndarray]:
    """Wirtinger gradient ``dE/dconj(AL[site]) = (H_AC(AC) - lambda AC) C^H`` of the
    normalised energy of the uniform MPS generated by ``AL``."""
    out = []
    for l in range(len(psi)):
        AC = psi.AC[l]
        y = ac_apply(envs.lefts[l], H[l], envs.rights[l], AC)
        lam = np.vdot(AC, y) / np.vdot(AC, AC)
        Dl, d, Dr = AC.shape
        g = freshape(y - lam * AC, (Dl * d, Dr)) @ psi.C[l].conj().T
        out.append(np.asfortranarray(freshape(g, (Dl, d, Dr))))
    return out


# --------------------------------------------------------------------------
# Algorithms  (vumps.jl, tdvp.jl, idmrg.jl, algdefs.jl)
# --------------------------------------------------------------------------
@dataclass
class VUMPS:
    """``VUMPS`` (``src/algorithms/algdefs.jl:26-35``)."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    verbosity: int = Defaults.verbosity
    alg_gauge: object = field(default_factory=alg_gauge)
    alg_eigsolve: object = field(default_factory=alg_eigsolve)
    alg_environments: object = field(default_factory=alg_environments)
    finalize: Optional[Callable] = None


@dataclass
class IDMRG:
    """``IDMRG`` (``src/algorithms/algdefs.jl:72-82``)."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    verbosity: int = Defaults.verbosity
    alg_gauge: object = field(default_factory=alg_gauge)
    alg_environments: object = field(default_factory=alg_environments)
    alg_eigsolve: object = field(default_factory=alg_eigsolve)
    finalize: Optional[Callable] = None


@dataclass
class TDVP:
    """``TDVP`` (``src/algorithms/algdefs.jl:167-173``)."""
    integrator: dict = field(default_factory=alg_expsolve)
    alg_gauge: object = field(default_factory=alg_gauge)
    verbosity: int = Defaults.verbosity
    finalize: Optional[Callable] = None


def _eig_params(alg):
    a = alg.alg if isinstance(alg, DynamicTol) else alg
    return a


def find_groundstate(psi0: CanonicalIMPS, H: SchurMPO, alg: VUMPS, envs: Optional[DMRGCache] = None,
                     log: Optional[list] = None):
    """``find_groundstate(psi0, H, ::VUMPS)`` (``src/algorithms/groundstates/vumps.jl:51-85``).

    Returns ``(psi, envs, info)`` with ``info = dict(niter, converged, losses, itererr)``.
    """
    psi = psi0.copy()
    if envs is None:
        envs = build_envs(psi, H)
    eps = calc_galerkin(psi, H, envs)
    ae = updatetol(alg.alg_environments, 0, eps)
    envs = build_envs(psi, H, tol=ae["tol"], maxiter=ae["maxiter"], init=envs)
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        psi, envs, eps = vumps_iteration(psi, H, envs, alg, it, eps)
        losses.append(eps)
        if log is not None:
            log.append(dict(iter=it, eps=eps, f=expectationvalue(psi, H, envs)))
        if eps <= alg.tol:
            converged = True
            break
    return psi, envs, dict(niter=it, converged=converged, losses=losses, itererr=losses[-1])


def vumps_iteration(psi: CanonicalIMPS, H: SchurMPO, envs: DMRGCache, alg: VUMPS, it: int, eps: float):
    """One pass of the ``find_groundstate(::VUMPS)`` loop (``vumps.jl:51-85``) at outer
    iteration ``it`` (1-based) after a Galerkin error ``eps``: ``localupdate_step!``
    (``vumps.jl:7-19``), ``gauge_step!`` (``:23-31``), ``recalculate!`` and
    ``calc_galerkin``.  Returns ``(psi, envs, eps_new)``."""
    N = len(psi)
    siter = it - 1
    ea = updatetol(alg.alg_eigsolve, siter, eps)
    ALs = []
    for site in range(N):
        GL, W, GR = envs.lefts[site], H[site], envs.rights[site]
        _, AC, _ = lanczos_eigsolve(lambda x: ac_apply(GL, W, GR, x), psi.AC[site], ea["tol"],
                                    ea["krylovdim"], ea["maxiter"], ea["eager"])
        GLc = envs.lefts[(site + 1) % N]
        _, C, _ = lanczos_eigsolve(lambda x: c_apply(GLc, GR, x), psi.C[site], ea["tol"],
                                   ea["krylovdim"], ea["maxiter"], ea["eager"])
        ALs.append(regauge(AC, C))
    ag = updatetol(alg.alg_gauge, siter, eps)
    psi = canonical_from_AL_keepAL(ALs, psi.C[N - 1], ag["tol"], ag["maxiter"])
    ae = updatetol(alg.alg_environments, siter, eps)
    envs = build_envs(psi, H, tol=ae["tol"], maxiter=ae["maxiter"], init=envs)
    if alg.finalize is not None:
        psi, envs = alg.finalize(it, psi, H, envs)
    return psi, envs, calc_galerkin(psi, H, envs)


def canonical_from_AL_keepAL(ALs, C0, tol, maxiter) -> CanonicalIMPS:
    """``gauge_step!`` (``vumps.jl:23-31``): keep the candidate ``AL``, right gauge fix
    from ``C0`` for ``AR, C``, then ``AC = AL C``."""
    psi = gaugefix(ALs, C0, order="R", tol=tol, maxiter=maxiter)
    psi.AC = [_mulAL(psi.AL[i], psi.C[i]) for i in range(len(ALs))]
    return psi


def timestep(psi: CanonicalIMPS, H: SchurMPO, dt: complex, alg: TDVP = None,
             envs: Optional[DMRGCache] = None):
    """``timestep(psi, H, dt, TDVP(), envs)`` (``src/algorithms/timeevo/tdvp.jl:34-53``)."""
    alg = alg or TDVP()
    if envs is None:
        envs = build_envs(psi, H)
    N = len(psi)
    ig = alg.integrator
    ACs, Cs = [], []
    for loc in range(N):
        GL, W, GR = envs.lefts[loc], H[loc], envs.rights[loc]
        ac, _ = exponentiate(lambda x: ac_apply(GL, W, GR, x), dt, psi.AC[loc], ig["tol"], ig["krylovdim"], ig["maxiter"])
        GLc = envs.lefts[(loc + 1) % N]
        c, _ = exponentiate(lambda x: c_apply(GLc, GR, x), dt, psi.C[loc], ig["tol"], ig["krylovdim"], ig["maxiter"])
        ACs.append(ac)
        Cs.append(c)
    ALs = [regauge(ACs[i], Cs[i]) for i in range(N)]
    g = alg.alg_gauge.alg if isinstance(alg.alg_gauge, DynamicTol) else alg.alg_gauge
    psi2 = canonical_from_AL(ALs, psi.C[N - 1], g["tol"], g["maxiter"])
    envs2 = build_envs(psi2, H, init=envs)
    return psi2, envs2


def time_evolve(psi0: CanonicalIMPS, H: SchurMPO, t_span: Sequence[complex], alg: TDVP = None,
                envs: Optional[DMRGCache] = None, observer: Optional[Callable] = None):
    """``time_evolve`` (``tdvp.jl:91-113``)."""
    alg = alg or TDVP()
    psi = psi0.copy()
    if envs is None:
        envs = build_envs(psi, H)
    hist = [observer(psi, 0, t_span[0]) if observer else expectationvalue(psi, H, envs)]
    for it in range(1, len(t_span)):
        dt = t_span[it] - t_span[it - 1]
        psi, envs = timestep(psi, H, dt, alg, envs)
        if alg.finalize is not None:
            psi, envs = alg.finalize(t_span[it - 1], psi, H, envs)
        hist.append(observer(psi, it, t_span[it]) if observer else expectationvalue(psi, H, envs))
    return psi, envs, hist


def idmrg_groundstate(psi0: CanonicalIMPS, H: SchurMPO, alg: IDMRG, envs: Optional[DMRGCache] = None):
    """``find_groundstate(psi0, H, ::IDMRG)`` (``src/algorithms/groundstates/idmrg.jl:12-82``)."""
    psi = psi0.copy()
    N = len(psi)
    if envs is None:
        envs = build_envs(psi, H)
    lefts = [x.copy(order="F") for x in envs.lefts]
    rights = [x.copy(order="F") for x in envs.rights]
    envs = DMRGCache(lefts, rights)
    eps = calc_galerkin(psi, H, envs)
    E = expectationvalue(psi, H, envs)
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        ea = updatetol(alg.alg_eigsolve, it - 1, eps)
        C_old = psi.C[N - 1].copy()
        for pos in range(N):
            GL, W, GR = envs.lefts[pos], H[pos], envs.rights[pos]
            _, ac, _ = lanczos_eigsolve(lambda x: ac_apply(GL, W, GR, x), psi.AC[pos], ea["tol"],
                                        ea["krylovdim"], ea["maxiter"], ea["eager"])
            Dl, d, Dr = ac.shape
            Q, R = qrpos(freshape(ac, (Dl * d, Dr)))
            psi.AL[pos] = np.asfortranarray(freshape(Q, (Dl, d, Dr)))
            psi.C[pos] = R
            psi.AC[pos] = psi.AL[pos].copy(order="F") if pos != N - 1 else ac
            nxt = (pos + 1) % N
            envs.lefts[nxt] = push_mpo_left(envs.lefts[pos], H[pos], psi.AL[pos])
        Enew = None
        for pos in range(N - 1, -1, -1):
            GL, W, GR = envs.lefts[pos], H[pos], envs.rights[pos]
            Enew, ac, _ = lanczos_eigsolve(lambda x: ac_apply(GL, W, GR, x), psi.AC[pos], ea["tol"],
                                           ea["krylovdim"], ea["maxiter"], ea["eager"])
            Dl, d, Dr = ac.shape
            Lf, Q = lqpos(freshape(ac, (Dl, d * Dr)))
            psi.C[pos - 1] = Lf
            psi.AR[pos] = np.asfortranarray(freshape(Q, (Dl, d, Dr)))
            psi.AC[pos] = psi.AR[pos].copy(order="F") if pos != 0 else ac
            prv = (pos - 1) % N
            envs.rights[prv] = push_mpo_right(envs.rights[pos], H[pos], psi.AR[pos])
        eps = _fnorm(psi.C[N - 1] - C_old)
        losses.append(eps)
        E = Enew
        if eps <= alg.tol:
            converged = True
            break
    ag = updatetol(alg.alg_gauge, it, eps)
    psi2 = canonical_from_sites([psi.AR[l] for l in range(N)], tol=ag["tol"], maxiter=ag["maxiter"])
    envs2 = build_envs(psi2, H, init=envs)
    return psi2, envs2, dict(niter=it, converged=converged, losses=losses, itererr=losses[-1], E=E)


# --------------------------------------------------------------------------
# Dense-MPO channel, correlators and entanglement (src/algorithms/groundstates/envs.jl:34-99,
# 284-304, 559-584; src/observables/expval.jl:60-79; src/observables/correlators.jl:13-42;
# src/observables/toolbox.jl:9-25)
# --------------------------------------------------------------------------
def dominant_env(psi: CanonicalIMPS, W: Optional[Sequence[np.ndarray]] = None, side: str = "left",
                 tol: float = Defaults.tol, krylovdim: int = Defaults.krylovdim, maxiter: int = Defaults.maxiter):
    """``dominant_env([W,] psi; side)`` (``envs.jl:34-99``): dominant (``:LM``) eigenvector of
    the identity (``W is None``, ``AL``/``AR`` pushes) or dense-MPO transfer matrix of one unit
    cell, from ``v0 = ones``, returned as ``(lambda, L)`` with ``L`` of shape
    ``(D, w, D)`` (``w = 1`` for the identity channel) and unit Frobenius norm."""
    N = len(psi)
    D = psi.AL[0].shape[0]
    w = 1 if W is None else W[0].shape[0]

    def tm(v):
        L = v
        if W is None:
            if side == "left":
                for l in range(N):
                    L = push_env_left(L, psi.AL[l])
            else:
                for l in range(N - 1, -1, -1):
                    L = push_env_right(L, psi.AR[l])
            return L
        if side == "left":
            for l in range(N):
                L = push_mpo_left(L, W[l], psi.AL[l])
        else:
            for l in range(N - 1, -1, -1):
                L = push_mpo_right(L, W[l], psi.AR[l])
        return L
    shape = (D, D) if W is None else (D, w, D)
    v0 = np.ones(shape, dtype=C128, order="F")
    lam, vec, _ = arnoldi_dominant(tm, v0, tol, krylovdim, maxiter, eager=True)
    L = freshape(np.asarray(vec), (D, w, D))
    return lam, np.asfortranarray(L / np.linalg.norm(L))


def normalize_envs(envs: "DMRGCache", psi: CanonicalIMPS) -> "DMRGCache":
    """``normalize_envs!(envs, below, operator, above)`` (``envs.jl:559-584``): every right
    environment to unit norm, then ``lefts[i+1] /= <C_i, H_C(i) C_i>``."""
    N = len(psi)
    for i in range(N):
        nr = np.linalg.norm(envs.rights[i])
        if nr > 0:
            envs.rights[i] = envs.rights[i] / nr
        lam = np.vdot(psi.C[i], c_apply(envs.lefts[(i + 1) % N], envs.rights[i], psi.C[i]))
        if abs(lam) > 0:
            envs.lefts[(i + 1) % N] = envs.lefts[(i + 1) % N] / lam
    return envs


def build_envs_dense(psi: CanonicalIMPS, W: Sequence[np.ndarray], tol: float = Defaults.tol,
                     krylovdim: int = Defaults.krylovdim, maxiter: int = Defaults.maxiter) -> "DMRGCache":
    """``DMRGCache(psi, ::DenseIMPO)`` (``envs.jl:284-304``): dominant left / right environments
    of the dense-MPO transfer matrix, pushed around the unit cell, then ``normalize_envs``."""
    N = len(psi)
    _, L0 = dominant_env(psi, W, "left", tol, krylovdim, maxiter)
    _, R0 = dominant_env(psi, W, "right", tol, krylovdim, maxiter)
    lefts = [None] * N
    rights = [None] * N
    lefts[0] = L0
    for l in range(1, N):
        lefts[l] = push_mpo_left(lefts[l - 1], W[l - 1], psi.AL[l - 1])
    rights[N - 1] = R0
    for l in range(N - 2, -1, -1):
        rights[l] = push_mpo_right(rights[l + 1], W[l + 1], psi.AR[l + 1])
    return normalize_envs(DMRGCache(lefts, rights), psi)


def expectationvalue_dense(psi: CanonicalIMPS, W: Sequence[np.ndarray], envs: "DMRGCache") -> complex:
    """``expectationvalue(psi, ::DenseIMPO, envs)`` (``expval.jl:60-79``): the sum over the unit
    cell of ``contract_mpo_expval(AC_i, GL_i, W_i, GR_i) = <AC_i, H_AC(i) AC_i>``, divided by
    ``<psi|psi>``."""
    N = len(psi)
    E = 0j
    for i in range(N):
        E += np.vdot(psi.AC[i], ac_apply(envs.lefts[i], W[i], envs.rights[i], psi.AC[i]))
    return E / state_dot(psi, psi)


def apply_local(O: np.ndarray, A: np.ndarray) -> np.ndarray:
    """``A'[a, u, b] = sum_s O[u, s] A[a, s, b]``."""
    return np.asfortranarray(np.einsum("us,asb->aub", O, A))


def correlator(psi: CanonicalIMPS, O1: np.ndarray, O2: np.ndarray, i: int, js: Sequence[int]) -> np.ndarray:
    """``correlator(psi, O1, O2, i, js)`` (``correlators.jl:13-42``): ``<O1_i O2_j> / <psi|psi>``
    for every ``j`` in ``js`` (1-based sites, increasing, ``j > i``).  As in the reference,
    the identity transfer through ``AR`` runs over sites ``ctr+1 .. j-1`` with ``ctr`` the
    previously evaluated ``j`` (the reference sets ``ctr = j`` after each value)."""
    N = len(psi)
    js = list(js)
    if js[0] <= i:
        raise ValueError("i should be smaller than j")
    AC = psi.AC[(i - 1) % N]
    V = push_env_left(np.eye(AC.shape[0], dtype=C128), apply_local(O1, AC), AC)
    out = np.zeros(len(js), dtype=C128)
    ctr = i
    for k, j in enumerate(js):
        for l in range(ctr + 1, j):
            A = psi.AR[(l - 1) % N]
            V = push_env_left(V, A, A)
        AR = psi.AR[(j - 1) % N]
        E = push_env_left(V, apply_local(O2, AR), AR)
        out[k] = np.trace(E)
        ctr = j
    return out / state_dot(psi, psi)


def entanglement_spectrum(psi: CanonicalIMPS, loc: int = 1) -> np.ndarray:
    """``entanglement_spectrum(psi, loc)`` (``toolbox.jl:9-14``): squared singular values of
    ``C[loc]`` (1-based bond, periodic), normalised, descending."""
    N = len(psi)
    s = np.linalg.svd(psi.C[(loc - 1) % N], compute_uv=False)
    p = np.abs(s) ** 2
    return np.sort(p / p.sum())[::-1]


def renyi_entropy(p: np.ndarray, alpha: float = 1.0) -> float:
    """von Neumann (``alpha = 1``) or Renyi entropy of a probability vector (natural log)."""
    p = np.asarray(p, dtype=float)
    p = p[p > 0]
    if alpha == 1:
        return float(-np.sum(p * np.log(p)))
    return float(np.log(np.sum(p ** alpha)) / (1.0 - alpha))


def entropy(psi: CanonicalIMPS, loc: int = 1, alpha: float = 1.0) -> float:
    """``entropy(psi, loc; alpha)`` (``toolbox.jl:16-25``)."""
    return renyi_entropy(entanglement_spectrum(psi, loc), alpha)


# --------------------------------------------------------------------------
# Time-evolution MPOs W^I / W^II (src/algorithms/timeevo/w1w2.jl:26-45).  The per-site
# kernel lives in the unvendored FiniteMPSAlgorithms package; this restates the
# published construction (Zaletel, Mong, Karrasch, Moore, Pollmann, PRB 91, 165112
# (2015), arXiv:1407.1832), which the reference cites.  Parity unpinned: only the
# physics (exp(delta H) to first order, the W^II error O(delta^2)) pins it.
# --------------------------------------------------------------------------
def _schur_blocks(W: np.ndarray):
    """Schur pieces of one site tensor W (m, d, n, d): D = W[0,:,n-1,:], C_b = W[0,:,b,:]
    (b interior), B_a = W[a,:,n-1,:], A_ab = W[a,:,b,:]."""
    m, n = W.shape[0], W.shape[2]
    D = W[0, :, n - 1, :]
    C = [W[0, :, b, :] for b in range(1, n - 1)]
    B = [W[a, :, n - 1, :] for a in range(1, m - 1)]
    A = [[W[a, :, b, :] for b in range(1, n - 1)] for a in range(1, m - 1)]
    return D, C, B, A


def timeevompo_site(W: np.ndarray, delta: complex, alg: str = "WII") -> np.ndarray:
    """W^I / W^II tensor of one Schur site tensor (m, d, n, d) -> (m-1, d, n-1, d).

    Level 0 of the result carries D, levels 1.. the interior channels:
    ``WI = [[1 + delta D, s C], [s B, A]]`` and for W^II, for every interior pair (a, b),
    the first block column of ``exp(M)`` with M the 4 x 4 block operator on the
    auxiliary states (0, c, b, bc): ``M[x, x] = delta D``, ``M[c, 0] = s C_b``,
    ``M[b, 0] = s B_a``, ``M[bc, 0] = A_ab``, ``M[bc, c] = s B_a``, ``M[bc, b] = s C_b``,
    ``s = sqrt(delta)``; ``W_D = E[0,0]``, ``W_C(b) = E[c,0]``, ``W_B(a) = E[b,0]``,
    ``W_A(a,b) = E[bc,0]``."""
    import scipy.linalg as sl
    d = W.shape[1]
    D, C, B, A = _schur_blocks(W)
    kl, kr = len(B), len(C)
    s = np.sqrt(complex(delta))
    out = np.zeros((kl + 1, d, kr + 1, d), dtype=C128, order="F")
    if alg == "WI":
        out[0, :, 0, :] = np.eye(d) + delta * D
        for b in range(kr):
            out[0, :, b + 1, :] = s * C[b]
        for a in range(kl):
            out[a + 1, :, 0, :] = s * B[a]
            for b in range(kr):
                out[a + 1, :, b + 1, :] = A[a][b]
        return out
    Z = np.zeros((d, d), dtype=C128)

    def block_exp(Cb, Ba, Aab):
        M = np.zeros((4 * d, 4 * d), dtype=C128)
        for x in range(4):
            M[x * d:(x + 1) * d, x * d:(x + 1) * d] = delta * D
        M[1 * d:2 * d, 0:d] = s * Cb
        M[2 * d:3 * d, 0:d] = s * Ba
        M[3 * d:4 * d, 0:d] = Aab
        M[3 * d:4 * d, 1 * d:2 * d] = s * Ba
        M[3 * d:4 * d, 2 * d:3 * d] = s * Cb
        E = sl.expm(M)
        return [E[x * d:(x + 1) * d, 0:d] for x in range(4)]
    out[0, :, 0, :] = block_exp(Z, Z, Z)[0]
    for b in range(kr):
        out[0, :, b + 1, :] = block_exp(C[b], Z, Z)[1]
    for a in range(kl):
        out[a + 1, :, 0, :] = block_exp(Z, B[a], Z)[2]
        for b in range(kr):
            out[a + 1, :, b + 1, :] = block_exp(C[b], B[a], A[a][b])[3]
    return out


def timeevompo(H: SchurMPO, delta: complex, alg: str = "WII") -> List[np.ndarray]:
    """``timeevompo(H::SparseIMPO, delta, WI()/WII())`` (``w1w2.jl:26-31``): the per-site
    tensors of the dense time-evolution MPO approximating ``exp(delta H)``."""
    return [timeevompo_site(W, delta, alg) for W in H.Ws]


def mpo_ring(Ws: Sequence[np.ndarray], L: int) -> np.ndarray:
    """Periodic-trace operator of an MPO on a ring of L sites (the MPO tensors repeated):
    sum over the bond indices of W_1 W_2 ... W_L, a d^L x d^L matrix (site 1 slowest)."""
    N = len(Ws)
    W0 = Ws[0]
    m, d = W0.shape[0], W0.shape[1]
    # T[i, (out), (in), j]: running product with open first and last bonds
    T = np.transpose(W0, (0, 1, 3, 2))  # (i, u, s, j)
    for l in range(1, L):
        Wl = Ws[l % N]
        T = np.einsum("iabk,kuvj->iaubvj", T, np.transpose(Wl, (0, 1, 3, 2)))
        i_, a, u, b, v, j = T.shape
        T = T.reshape(i_, a * u, b * v, j)
    return np.einsum("iabi->ab", T)


# --------------------------------------------------------------------------
# Two-site IDMRG (IDMRG2): src/algorithms/groundstates/idmrg.jl:90-235 and the two-site
# effective Hamiltonian src/algorithms/groundstates/effective.jl:113-197.  Sites 0-based
# (reference site pos = p + 1); the truncation is ``truncdim(D)`` (keep at most D
# singular values), the reference's ``tsvd`` + ``normalize!(s)`` split.
# --------------------------------------------------------------------------
@dataclass
class IDMRG2:
    """``IDMRG2`` (``src/algorithms/algdefs.jl:106-116``) with ``trunc = truncdim(D)``."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    alg_gauge: object = field(default_factory=alg_gauge)
    alg_eigsolve: object = field(default_factory=alg_eigsolve)


def ac2_apply(GL, W1, W2, GR, x):
    """``MPO_AC2_Hamiltonian`` action (``effective.jl:160-197``):
    ``y[b,u1,u2,c] = sum GL[b,w1,a] x[a,s1,s2,bb] W1[w1,u1,w2,s1] W2[w2,u2,wr,s2] GR[bb,wr,c]``."""
    Dl, d1, d2, Dr = x.shape
    m = W1.shape[0]
    T1 = freshape(freshape(GL, (Dl * m, Dl)) @ freshape(x, (Dl, d1 * d2 * Dr)), (Dl, m, d1, d2, Dr))
    T2 = np.tensordot(T1, W1, axes=([1, 2], [0, 3]))        # [b, s2, bb, u1, w2]
    T3 = np.tensordot(T2, W2, axes=([4, 1], [0, 3]))        # [b, bb, u1, u2, wr]
    return np.asfortranarray(np.tensordot(T3, GR, axes=([1, 4], [0, 1])))


def ac2(psi: CanonicalIMPS, p: int, kind: str = "ACAR") -> np.ndarray:
    """``AC2(psi, pos; kind)`` (``effective.jl:138-152``), 0-based ``p`` (periodic)."""
    N = len(psi)
    p %= N
    q = (p + 1) % N
    A1, A2 = (psi.AC[p], psi.AR[q]) if kind == "ACAR" else (psi.AL[p], psi.AC[q])
    return np.asfortranarray(np.einsum("asm,mtb->astb", A1, A2))


def idmrg2_split(x2: np.ndarray, D: int):
    """``_idmrg2_split`` (``idmrg.jl:107-111``): SVD of the (Dl d1) x (d2 Dr) matrix, the
    ``D`` largest values kept and normalised; returns ``(al, c, ar)``."""
    Dl, d1, d2, Dr = x2.shape
    U, S, Vh = np.linalg.svd(freshape(x2, (Dl * d1, d2 * Dr)), full_matrices=False)
    k = min(D, len(S))
    s = S[:k] / np.linalg.norm(S[:k])
    al = np.asfortranarray(freshape(U[:, :k], (Dl, d1, k)))
    ar = np.asfortranarray(freshape(Vh[:k, :], (k, d2, Dr)))
    return al, np.diag(s).astype(C128), ar


def _div_tail(A, C):
    """``A / C`` on the last bond (``X C = A``)."""
    Dl, d, Dr = A.shape
    Xm = np.linalg.solve(C.T, freshape(A, (Dl * d, Dr)).T).T
    return np.asfortranarray(freshape(Xm, (Dl, d, C.shape[1])))


def _frontdiv(C, A):
    """``C \\ A`` on the first bond."""
    Dl, d, Dr = A.shape
    Xm = np.linalg.solve(C, freshape(A, (Dl, d * Dr)))
    return np.asfortranarray(freshape(Xm, (C.shape[1], d, Dr)))


def idmrg2_sweep(psi: CanonicalIMPS, H: SchurMPO, envs: DMRGCache, ea: dict, D: int):
    """``_localupdate_sweep_idmrg2!`` (``idmrg.jl:113-185``); returns ``(C_old, E)``."""
    N = len(psi)
    AL, AR, Cs, AC = psi.AL, psi.AR, psi.C, psi.AC

    def tl(s):
        s %= N
        envs.lefts[s] = push_mpo_left(envs.lefts[s - 1], H[s - 1], AL[s - 1])

    def tr(s):
        s %= N
        q = (s + 1) % N
        envs.rights[s] = push_mpo_right(envs.rights[q], H[q], AR[q])

    def solve(p, kind):
        q = (p + 1) % N
        GL, W1, W2, GR = envs.lefts[p % N], H[p % N], H[q], envs.rights[q]
        E, x, _ = lanczos_eigsolve(lambda v: ac2_apply(GL, W1, W2, GR, v), ac2(psi, p, kind), ea["tol"],
                                   ea["krylovdim"], ea["maxiter"], ea["eager"])
        return E, x

    for p in range(N - 1):
        _, x = solve(p, "ACAR")
        al, c, ar = idmrg2_split(x, D)
        AL[p], Cs[p], AR[p + 1] = al, c, ar
        AC[p + 1] = _mulCA(c, ar)
        tl(p + 1)
        tr(p)
    AL[N - 1] = _div_tail(AC[N - 1], Cs[N - 1])
    AC[0] = _mulAL(AL[0], Cs[0])
    _, x = solve(N - 1, "ALAC")
    al, c, ar = idmrg2_split(x, D)
    AL[N - 1], Cs[N - 1], AR[0] = al, c, ar
    AC[N - 1] = _mulAL(al, c)
    AC[0] = _mulCA(c, ar)
    AL[0] = _div_tail(AC[0], Cs[0])
    C_old = c.copy()
    tl(0)
    tr(N - 1)
    for p in range(N - 2, -1, -1):
        _, x = solve(p, "ALAC")
        al, c, ar = idmrg2_split(x, D)
        AL[p] = al
        AC[p] = _mulAL(al, c)
        Cs[p] = c
        AR[p + 1] = ar
        AC[p + 1] = _mulCA(c, ar)
        tl(p + 1)
        tr(p)
    AC[N - 1] = _mulCA(Cs[N - 2], AR[N - 1])
    AR[0] = _frontdiv(Cs[N - 1], AC[0])
    E, x = solve(N - 1, "ACAR")
    al, c, ar = idmrg2_split(x, D)
    AL[N - 1], Cs[N - 1], AR[0] = al, c, ar
    AR[N - 1] = _frontdiv(Cs[N - 2], _mulAL(al, c))
    AC[0] = _mulCA(c, ar)
    tl(0)
    tr(N - 1)
    return C_old, E


def idmrg2_groundstate(psi0: CanonicalIMPS, H: SchurMPO, alg: IDMRG2, envs: Optional[DMRGCache] = None):
    """``find_groundstate(psi0, H, ::IDMRG2)`` (``idmrg.jl:203-235``)."""
    psi = psi0.copy()
    N = len(psi)
    if N < 2:
        raise ValueError("IDMRG2 requires unit cell length >= 2")
    if envs is None:
        envs = build_envs(psi, H)
    envs = DMRGCache([x.copy(order="F") for x in envs.lefts], [x.copy(order="F") for x in envs.rights])
    eps = calc_galerkin(psi, H, envs)
    losses = [eps]
    converged = False
    it = 0
    E = None
    for it in range(1, alg.maxiter + 1):
        ea = updatetol(alg.alg_eigsolve, it - 1, eps)
        C_old, E = idmrg2_sweep(psi, H, envs, ea, alg.D)
        eps = _fnorm(psi.C[N - 1] - C_old)
        losses.append(eps)
        if eps <= alg.tol:
            converged = True
            break
    ag = updatetol(alg.alg_gauge, it, eps)
    psi2 = canonical_from_sites([psi.AR[l] for l in range(N)], tol=ag["tol"], maxiter=ag["maxiter"])
    envs2 = build_envs(psi2, H)
    return psi2, envs2, dict(niter=it, converged=converged, losses=losses, itererr=losses[-1], E=E)


# --------------------------------------------------------------------------
# MPO application mult(W, psi, VOMPS(D)): src/algorithms/arithmetics/mult.jl (MultCache
# :58-197, local maps :226-230 / :294-303 / :705-716, calc_galerkin :586-593, mult :794-806,
# svdguess_mult :848-870), compression_sweeps!(::VOMPS) (arithmetics/envs.jl:51-93), the
# lazy SVD guess (arithmetics/compress.jl:161-190) and the ternary pushes
# (src/transfermatrix.jl:77-107).  W is a dense MPO (list of (wl, u, wr, d) tensors, the
# DenseIMPO channel: operator.AL = AR = AC = W, operator.C = identity).
# --------------------------------------------------------------------------
@dataclass
class VOMPS:
    """``VOMPS(; D, tol, maxiter, verbosity, alg_gauge, alg_environments, alg_orth)``
    (``src/algorithms/algdefs.jl:118-153``)."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    alg_gauge: object = field(default_factory=alg_gauge)
    alg_environments: object = field(default_factory=alg_environments)


def push_ternary_left(L, below, W, above):
    """``L'[bl',w',al'] = sum conj(below[bl,u,bl']) L[bl,w,al] W[w,u,w',d] above[al,d,al']``
    (``transfermatrix.jl:77-82``); ``L`` is ``(below bond, w, above bond)``."""
    Db, du, Dbr = below.shape
    Da, dd, Dar = above.shape
    w, wr = W.shape[0], W.shape[2]
    T1 = freshape(freshape(L, (Db * w, Da)) @ freshape(above, (Da, dd * Dar)), (Db, w, dd, Dar))
    T2 = np.asfortranarray(np.einsum("wuvd,bwdc->buvc", W, T1, optimize=True))
    out = freshape(below, (Db * du, Dbr)).conj().T @ freshape(T2, (Db * du, wr * Dar))
    return np.asfortranarray(freshape(out, (Dbr, wr, Dar)))


def push_ternary_right(R, above, W, below):
    """``R'[al',w',bl'] = sum above[al',d,al] R[al,w,bl] W[w',u,w,d] conj(below[bl',u,bl])``
    (``transfermatrix.jl:94-99``); ``R`` is ``(above bond, w, below bond)``."""
    Dal, dd, Da = above.shape
    Dbl, du, Db = below.shape
    wl, w = W.shape[0], W.shape[2]
    T1 = freshape(freshape(above, (Dal * dd, Da)) @ freshape(R, (Da, w * Db)), (Dal, dd, w, Db))
    T2 = np.asfortranarray(np.einsum("vuwd,adwb->avub", W, T1, optimize=True))
    out = freshape(T2, (Dal * wl, du * Db)) @ freshape(below, (Dbl, du * Db)).conj().T
    return np.asfortranarray(freshape(out, (Dal, wl, Dbl)))


def mult_ac(GL, W, GR, x):
    """``_mapAC`` (``mult.jl:226-230``): ``y[aL,u,aR] = sum GL[aL,w,bL] x[bL,s,bR] W[w,u,w',s]
    GR[bR,w',aR]`` with ``GL (below, w, above)``, ``GR (above, w', below)``."""
    Db, w, Da = GL.shape
    _, d, Dar = x.shape
    wr, Dbr = W.shape[2], GR.shape[2]
    T1 = freshape(freshape(GL, (Db * w, Da)) @ freshape(x, (Da, d * Dar)), (Db, w, d, Dar))
    T2 = np.asfortranarray(np.einsum("wuvs,bwsc->bucv", W, T1, optimize=True))
    y = freshape(T2, (Db * W.shape[1], Dar * wr)) @ freshape(GR, (Dar * wr, Dbr))
    return np.asfortranarray(freshape(y, (Db, W.shape[1], Dbr)))


def mult_c(GL, GR, C):
    """``_mapC`` with the identity operator bond weight (``mult.jl:705-716``):
    ``y[jL,jR] = sum GL[jL,w,w2] C[w2,r2] GR[r2,w,jR]``."""
    Db, w, Da = GL.shape
    Dar, _, Dbr = GR.shape
    U = freshape(C @ freshape(GR, (Dar, w * Dbr)), (Da, w, Dbr))   # U[w2, w, jR]
    GLp = freshape(np.asfortranarray(GL.transpose(0, 2, 1)), (Db, Da * w))
    return np.asfortranarray(GLp @ freshape(np.asfortranarray(U), (Da * w, Dbr)))


def env_start_vector(n: int) -> np.ndarray:
    """Deterministic start of the environment eigensolves (the reference draws ``randn``):
    ``exp(2 pi i frac(k phi))``, ``phi`` the golden ratio conjugate, ``k = 0 .. n-1``."""
    k = np.arange(n, dtype=np.float64)
    ph = 2.0 * math.pi * np.mod(k * 0.6180339887498949, 1.0)
    return np.exp(1j * ph)


@dataclass
class MultCache:
    """``MultCache`` (``mult.jl:58-66``): ``lefts[l]`` ``(below, w, above)``, ``rights[l]``
    ``(above, w, below)`` of the ``<below|W|above>`` channel."""
    Ws: List[np.ndarray]
    bra: CanonicalIMPS
    ket: CanonicalIMPS
    lefts: List[np.ndarray]
    rights: List[np.ndarray]


def mixed_fixedpoints(below: CanonicalIMPS, Ws, above: CanonicalIMPS, tol: float, maxiter: int,
                      GL0=None, GR0=None, krylovdim: int = Defaults.krylovdim):
    """``mixed_fixedpoints`` (``mult.jl:93-158``): the :LM fixed points of the ternary transfer
    matrices, the other sites by pushes, GR Frobenius-normalised, then GL[l+1] divided by
    ``lambda_l = <below.C[l], mapC(GL[l+1], GR[l], above.C[l])>``."""
    N = len(below)
    Lw = len(Ws)
    Dl = below.AL[0].shape[0]
    Da = above.AL[0].shape[0]
    Dw = Ws[0].shape[0]

    def tleft(v):
        for l in range(N):
            v = push_ternary_left(v, below.AL[l], Ws[l % Lw], above.AL[l])
        return v

    def tright(v):
        for l in range(N - 1, -1, -1):
            v = push_ternary_right(v, above.AR[l], Ws[l % Lw], below.AR[l])
        return v
    v0L = GL0.copy(order="F") if GL0 is not None else freshape(env_start_vector(Dl * Dw * Da), (Dl, Dw, Da))
    _, vL, _ = arnoldi_dominant(tleft, v0L, tol, krylovdim, maxiter, eager=True)
    GLs = [None] * N
    GLs[0] = np.asfortranarray(freshape(np.asarray(vL), (Dl, Dw, Da)))
    for l in range(1, N):
        GLs[l] = push_ternary_left(GLs[l - 1], below.AL[l - 1], Ws[(l - 1) % Lw], above.AL[l - 1])
    v0R = GR0.copy(order="F") if GR0 is not None else freshape(env_start_vector(Da * Dw * Dl), (Da, Dw, Dl))
    _, vR, _ = arnoldi_dominant(tright, v0R, tol, krylovdim, maxiter, eager=True)
    GRs = [None] * N
    GRs[N - 1] = np.asfortranarray(freshape(np.asarray(vR), (Da, Dw, Dl)))
    for l in range(N - 2, -1, -1):
        GRs[l] = push_ternary_right(GRs[l + 1], above.AR[l + 1], Ws[(l + 1) % Lw], below.AR[l + 1])
    GRs = [g / _fnorm(g) for g in GRs]
    for l in range(N):
        nx = (l + 1) % N
        lam = np.vdot(below.C[l], mult_c(GLs[nx], GRs[l], above.C[l]))
        if lam == 0:
            raise ValueError(f"ternary environment: local overlap lambda = 0 at site {l + 1}")
        GLs[nx] = np.asfortranarray(GLs[nx] / lam)
    return GLs, GRs


def mult_local_ac(envs: MultCache, l: int):
    return mult_ac(envs.lefts[l], envs.Ws[l % len(envs.Ws)], envs.rights[l], envs.ket.AC[l])


def mult_local_c(envs: MultCache, l: int):
    N = len(envs.bra)
    return mult_c(envs.lefts[(l + 1) % N], envs.rights[l], envs.ket.C[l])


def mult_galerkin(envs: MultCache, x: CanonicalIMPS) -> float:
    """``calc_galerkin(envs::MultCache, x)`` (``mult.jl:586-593``) with ``_galerkin``
    (``mult.jl:278-284``)."""
    eps = 0.0
    for l in range(len(x)):
        ac = mult_local_ac(envs, l)
        ac = ac / _fnorm(ac)
        AL = x.AL[l]
        Dl, d, Dr = AL.shape
        A2 = freshape(AL, (Dl * d, Dr))
        x2 = freshape(ac, (Dl * d, Dr))
        eps = max(eps, _fnorm(x2 - A2 @ (A2.conj().T @ x2)))
    return eps


def _tsvd_rows(B: np.ndarray, D: int):
    """``tsvd(B, (1,), (2, 3); trunc = truncdim(D))``: ``B = u diag(s) v``, ``v`` (k, d2, d3)."""
    r, d2, d3 = B.shape
    U, S, Vh = np.linalg.svd(freshape(B, (r, d2 * d3)), full_matrices=False)
    k = min(D, len(S))
    return U[:, :k], S[:k], np.asfortranarray(freshape(Vh[:k, :], (k, d2, d3)))


def svdguess_mult_sites(Ws: Sequence[np.ndarray], ALs: Sequence[np.ndarray], D: int) -> List[np.ndarray]:
    """``svdguess_mult(Ws, ALs, D)`` (``mult.jl:853-870``) through ``_lazy_svd_guess``
    (``compress.jl:161-190``): the product's site tensors
    ``B[(wl, bl), u, (wr, br)] = sum_d W[wl,u,wr,d] AL[bl,d,br]`` (``operators/linalg.jl:15-20``)
    built right to left with the carry absorbed, each truncated to bond ``D``."""
    N = len(ALs)
    Lw = len(Ws)

    def site(i, carry):
        W4 = Ws[i % Lw]
        A = ALs[i]
        wl, u, wr, dd = W4.shape
        bl, _, br = A.shape
        if carry is None:
            B5 = np.einsum("wurd,bdc->wburc", W4, A, optimize=True)
            return np.asfortranarray(freshape(np.asfortranarray(B5), (wl * bl, u, wr * br)))
        f = carry.shape[1]
        l4 = freshape(carry, (wr, br, f))
        Tb = np.einsum("bdc,rcf->bdrf", A, l4, optimize=True)
        B3 = np.einsum("wurd,bdrf->wbuf", W4, Tb, optimize=True)
        return np.asfortranarray(freshape(np.asfortranarray(B3), (wl * bl, u, f)))

    out = [None] * N
    B = site(N - 1, None)
    carry = None
    for i in range(N - 1, 0, -1):
        u, s, v = _tsvd_rows(B, D)
        out[i] = v
        carry = np.asfortranarray(u * s)
        B = site(i - 1, carry)
    u, s, v = _tsvd_rows(B, D)
    out[0] = np.asfortranarray(s[:, None, None] * v)
    if N >= 2:
        out[N - 1] = np.asfortranarray(np.einsum("asb,bc->asc", out[N - 1], u, optimize=True))
    else:
        r1, s1, r2 = out[0].shape
        U2, S2, _ = np.linalg.svd(freshape(out[0], (r1 * s1, r2)), full_matrices=False)
        k2 = min(D, len(S2))
        out[0] = np.asfortranarray(freshape(U2[:, :k2] * S2[:k2], (r1, s1, k2)))
    return out


def mult_sweeps(envs: MultCache, alg: VOMPS):
    """``compression_sweeps!(envs::MultCache, alg::VOMPS)`` (``arithmetics/envs.jl:51-93``)."""
    x = envs.bra
    N = len(x)
    eps = mult_galerkin(envs, x)
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        ALs = [regauge(mult_local_ac(envs, l), mult_local_c(envs, l)) for l in range(N)]
        ag = updatetol(alg.alg_gauge, it - 1, eps)
        x = canonical_from_AL_keepAL(ALs, x.C[N - 1], ag["tol"], ag["maxiter"])
        ae = updatetol(alg.alg_environments, it - 1, eps)
        GLs, GRs = mixed_fixedpoints(x, envs.Ws, envs.ket, ae["tol"], ae["maxiter"],
                                     GL0=envs.lefts[0], GR0=envs.rights[N - 1])
        envs = MultCache(envs.Ws, x, envs.ket, GLs, GRs)
        eps = mult_galerkin(envs, x)
        losses.append(eps)
        if eps <= alg.tol:
            converged = True
            break
    return envs, dict(niter=it, converged=converged, losses=losses, itererr=losses[-1])


def mult(Ws: Sequence[np.ndarray], psi: CanonicalIMPS, alg: VOMPS):
    """``mult(W, psi, ::VOMPS)`` (``mult.jl:794-806``) for a dense MPO ``W``: initial state
    ``svdguess_mult(W, psi, alg.D)``, ternary environments at the initial ``alg_environments``
    tolerance, then ``compression_sweeps!``.  Returns ``(y, envs, info)``."""
    if len(psi) % len(Ws) != 0:
        raise ValueError("incompatible unit-cell lengths of MPS and MPO")
    x0 = canonical_from_sites(svdguess_mult_sites(Ws, psi.AL, alg.D))
    ae = alg.alg_environments
    base = ae.alg if isinstance(ae, DynamicTol) else ae
    GLs, GRs = mixed_fixedpoints(x0, list(Ws), psi, base["tol"], base["maxiter"])
    envs, info = mult_sweeps(MultCache(list(Ws), x0, psi, GLs, GRs), alg)
    return envs.bra, envs, info
