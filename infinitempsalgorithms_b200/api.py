"""Host-side mirror of the InfiniteMPSAlgorithms API for the VUMPS/TDVP inner loop.

Same names, argument meaning and error behaviour as the Julia reference
(``find_groundstate``, ``VUMPS``, ``IDMRG``, ``TDVP``, ``timestep``,
``time_evolve``, ``DMRGCache``, ``recalculate``, ``AC_hamiltonian``,
``C_hamiltonian``, ``calc_galerkin``, ``expectationvalue``), backed by the
sm_100a library through its C ABI.  Site indices are 1-based and periodic
(Julia ``mod1``), as in the reference.  Tensors are NumPy complex128 arrays
in the reference's index order; the device copies are column-major.
"""
from __future__ import annotations

import ctypes as C
import math
import weakref
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import check, cbuf, dptr, ptr_array

__all__ = [
    "Defaults", "DynamicTol", "updatetol", "Context", "default_context", "sigma", "spin", "mpohamiltonian",
    "SparseIMPO", "tfim_hamiltonian", "heisenberg_hamiltonian", "hubbard_hamiltonian", "PeriodicVector",
    "CanonicalIMPS", "randomimps", "random_site_tensors", "DMRGCache", "recalculate", "AC_hamiltonian",
    "C_hamiltonian", "fixedpoint", "integrate", "regauge", "calc_galerkin", "expectationvalue", "VUMPS",
    "IDMRG", "IDMRG2", "ac2_apply", "VOMPS", "MultCache", "svdguess_mult", "mult", "TDVP", "IterativeConvergenceInfo", "find_groundstate", "timestep", "time_evolve", "linsolve",
    "qrpos", "lqpos", "tsvd", "push_env_left", "push_env_right", "push_mpo_left", "push_mpo_right",
    "energy_gradient_mpo", "energy_gradient_AL", "coupling_gradient", "rrule_energy", "find_groundstate_batch",
    "DenseIMPO", "identityimpo", "timeevompo", "dominant_env", "correlator", "entanglement_spectrum", "renyi_entropy", "entropy",
]


# ---------------------------------------------------------------------------
# Defaults / DynamicTol (src/utility.jl:136-171, 297-365)
# ---------------------------------------------------------------------------
class Defaults:
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

    @staticmethod
    def alg_eigsolve(tol=1.0e-10, maxiter=300, krylovdim=30, eager=True, tol_factor=1.0e-3, dynamic=True):
        a = dict(tol=tol, maxiter=maxiter, krylovdim=krylovdim, eager=eager)
        return DynamicTol(a, Defaults.tol_min, Defaults.tol_max, tol_factor) if dynamic else a

    @staticmethod
    def alg_gauge(tol=1.0e-13, maxiter=300, dynamic=True):
        a = dict(tol=tol, maxiter=maxiter)
        return DynamicTol(a, Defaults.tol_min, Defaults.tol_max, Defaults.gauge_tolfactor) if dynamic else a

    @staticmethod
    def alg_environments(tol=1.0e-10, maxiter=300, dynamic=True):
        a = dict(tol=tol, maxiter=maxiter)
        return DynamicTol(a, Defaults.tol_min, Defaults.tol_max, Defaults.envs_tolfactor) if dynamic else a

    @staticmethod
    def alg_expsolve(tol=1.0e-10, maxiter=300, krylovdim=30):
        return dict(tol=tol, maxiter=maxiter, krylovdim=krylovdim)


@dataclass
class DynamicTol:
    """``DynamicTol(alg, tol_min, tol_max, tol_factor)``; raises ``ValueError``
    (the reference's ``ArgumentError``) unless ``0 <= tol_min <= tol_max``."""
    alg: dict
    tol_min: float = 1.0e-6
    tol_max: float = 1.0e-2
    tol_factor: float = 0.1

    def __post_init__(self):
        if not (0 <= self.tol_min <= self.tol_max):
            raise ValueError("DynamicTol requires 0 <= tol_min <= tol_max")


def updatetol(alg, iter: int, eps: float):
    """``updatetol``: ``clamp(eps * tol_factor / sqrt(max(iter, 1)), tol_min, tol_max)``."""
    if not isinstance(alg, DynamicTol):
        return alg
    it = max(iter, 1)
    out = dict(alg.alg)
    out["tol"] = min(max(eps * alg.tol_factor / math.sqrt(it), alg.tol_min), alg.tol_max)
    return out


def _unwrap(alg):
    return alg.alg if isinstance(alg, DynamicTol) else alg


# ---------------------------------------------------------------------------
# Device context
# ---------------------------------------------------------------------------
class Context:
    """One CUDA stream + library context (``imps_ctx``) on one device."""

    def __init__(self, device: int = 0, precision: int = L.IMPS_PREC_FP64, nslices: int = 5):
        self.lib = L.load()
        h = C.c_void_p()
        check(self.lib.imps_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self._children = weakref.WeakSet()
        self._mpo_links = []
        self.set_precision(precision, nslices)

    def _adopt(self, obj):
        self._children.add(obj)
        return obj

    def set_precision(self, mode: int, nslices: int = 5):
        check(self.lib.imps_ctx_set_precision(self.h, mode, nslices), self.h)
        self.precision = mode
        self.nslices = nslices

    def set_stream(self, stream_ptr: int):
        check(self.lib.imps_ctx_set_stream(self.h, C.c_void_p(stream_ptr)), self.h)

    def synchronize(self):
        check(self.lib.imps_ctx_synchronize(self.h), self.h)

    def profile(self, enable: bool = True):
        check(self.lib.imps_ctx_profile(self.h, int(enable)), self.h)

    def profile_classes(self, classes=None):
        """Time only these kernel classes (None: all)."""
        csv = ",".join(classes) if classes else None
        check(self.lib.imps_ctx_profile_classes(self.h, csv.encode() if csv else None), self.h)

    def profile_reset(self):
        check(self.lib.imps_ctx_profile_reset(self.h), self.h)

    def profile_get(self, cls: str):
        n = C.c_int64()
        ms = C.c_double()
        work = C.c_double()
        check(self.lib.imps_ctx_profile_get(self.h, cls.encode(), C.byref(n), C.byref(ms), C.byref(work)), self.h)
        return n.value, ms.value, work.value

    def profile_dump(self):
        """{class@site: (launches, total_ms, work)} for every kernel class timed so far."""
        buf = C.create_string_buffer(1 << 16)
        check(self.lib.imps_ctx_profile_dump(self.h, buf, len(buf)), self.h)
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms, work = line.split()
            out[name] = (int(n), float(ms), float(work))
        return out

    def counters(self):
        arr = (C.c_int64 * 11)()
        check(self.lib.imps_ctx_counters_ext(self.h, arr, 11), self.h)
        return dict(ac_apply=arr[0], c_apply=arr[1], push=arr[2], gemm=arr[3], kernels=arr[4], qr=arr[5],
                    gemm_flops=arr[6], qr_flops=arr[7], split_launches=arr[8], split_alg_flops=arr[9],
                    split_exec_ops=arr[10])

    def close(self):
        """Destroy the context; device objects created on it are released first."""
        if getattr(self, "h", None):
            for child in list(self._children) + self._mpo_links:
                child._release()
            self._mpo_links = []
            self.lib.imps_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ---------------------------------------------------------------------------
# Models (src/models.jl:61-122); Hubbard: Jordan-Wigner, 4 hopping channels
# ---------------------------------------------------------------------------
def sigma(which: str) -> np.ndarray:
    return {"x": np.array([[0, 1], [1, 0]], complex), "y": np.array([[0, -1j], [1j, 0]], complex),
            "z": np.array([[1, 0], [0, -1]], complex)}[which]


def spin(which: str) -> np.ndarray:
    return sigma(which) / 2


def mpohamiltonian(h1: np.ndarray, pairs: Sequence) -> np.ndarray:
    """Schur level matrix as the dense ``(n, d, n, d)`` tompotensor (``models.jl:82-100``)."""
    d = h1.shape[0]
    n = len(pairs) + 2
    W = np.zeros((n, d, n, d), complex, order="F")
    eye = np.eye(d)
    W[0, :, 0, :] = eye
    W[n - 1, :, n - 1, :] = eye
    W[0, :, n - 1, :] = h1
    for k, (coeff, a, b) in enumerate(pairs):
        W[0, :, k + 1, :] = coeff * np.asarray(a, complex)
        W[k + 1, :, n - 1, :] = np.asarray(b, complex)
    return W


class SparseIMPO:
    """Schur-form Hamiltonian MPO (``SparseIMPO``): site tensors ``(m, d, n, d)``."""

    def __init__(self, Ws: Sequence[np.ndarray]):
        if len(Ws) == 0:
            raise ValueError("Ws must not be empty")
        self.Ws = [cbuf(W) for W in Ws]
        N = len(self.Ws)
        for l in range(N):
            if self.Ws[l].shape[2] != self.Ws[(l + 1) % N].shape[0]:
                raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, "level chain mismatch")
        self._dev = {}

    def __len__(self):
        return len(self.Ws)

    def __getitem__(self, l: int):
        return self.Ws[(l - 1) % len(self.Ws)]

    def phydims(self):
        return [W.shape[1] for W in self.Ws]

    def handle(self, ctx: Context):
        key = id(ctx)
        if key not in self._dev:
            N = len(self.Ws)
            m = (C.c_int * N)(*[W.shape[0] for W in self.Ws])
            d = (C.c_int * N)(*[W.shape[1] for W in self.Ws])
            n = (C.c_int * N)(*[W.shape[2] for W in self.Ws])
            h = C.c_void_p()
            check(ctx.lib.imps_mpo_create(ctx.h, N, m, d, n, ptr_array(self.Ws), C.byref(h)), ctx.h)
            self._dev[key] = (ctx, h)
            ctx._mpo_links.append(_MpoHandle(self, key))
        return self._dev[key][1]

    def _release_key(self, key):
        ent = self._dev.pop(key, None)
        if ent is not None:
            ent[0].lib.imps_mpo_destroy(ent[1])

    def __del__(self):
        for key in list(getattr(self, "_dev", {})):
            try:
                self._release_key(key)
            except Exception:
                pass


class DenseIMPO(SparseIMPO):
    """``DenseIMPO``: a periodic string of dense MPO tensors ``(m, d, n, d)`` without the
    Schur structure (transfer matrices, time-evolution MPOs).  Its environments are
    the dominant fixed points of the MPO transfer matrix (``DMRGCache(psi, ::DenseIMPO)``,
    ``src/algorithms/groundstates/envs.jl:284-304``) and its expectation value is the
    sum of the local contractions (``src/observables/expval.jl:60-79``)."""


def identityimpo(dims: Sequence[int]) -> DenseIMPO:
    """The identity MPO (bond dimension 1) on a unit cell with physical dimensions ``dims``."""
    return DenseIMPO([np.eye(d, dtype=complex).reshape(1, d, 1, d) for d in dims])


class _MpoHandle:
    """Weak link from a context to an MPO's device copy on it (released with the context)."""

    def __init__(self, mpo, key):
        self.mpo = weakref.ref(mpo)
        self.key = key

    def _release(self):
        m = self.mpo()
        if m is not None:
            m._release_key(self.key)


def tfim_hamiltonian(J=1.0, h=1.0) -> SparseIMPO:
    """``H = -J sum sx sx - h sum sz`` (``src/models.jl:119-122``)."""
    return SparseIMPO([mpohamiltonian(-h * sigma("z"), [(-J, sigma("x"), sigma("x"))])])


def heisenberg_hamiltonian(J=1.0, Delta=1.0, h=0.0) -> SparseIMPO:
    """``H = J sum (SxSx + SySy + Delta SzSz) - h sum Sz`` (``src/models.jl:107-111``)."""
    Sx, Sy, Sz = spin("x"), spin("y"), spin("z")
    return SparseIMPO([mpohamiltonian(-h * Sz, [(J, Sx, Sx), (J, Sy, Sy), (J * Delta, Sz, Sz)])])


def hubbard_hamiltonian(t=1.0, U=4.0, mu=2.0) -> SparseIMPO:
    """Spinful Fermi-Hubbard chain (Jordan-Wigner, w = 6) on ``(|0>, |up>, |dn>, |updn>)``.

    ``H = -t sum_s (c+_{s,i} c_{s,i+1} + h.c.) + U sum n_up n_dn - mu sum n``; the
    hops are ``(c+_s P)(x)c_s`` and ``(P c_s)(x)c+_s`` with the parity ``P = (-1)^n``.
    """
    c_up = np.zeros((4, 4), complex)
    c_dn = np.zeros((4, 4), complex)
    c_up[0, 1] = 1.0
    c_up[2, 3] = 1.0
    c_dn[0, 2] = 1.0
    c_dn[1, 3] = -1.0
    P = np.diag([1.0, -1.0, -1.0, 1.0]).astype(complex)
    n = np.diag([0.0, 1.0, 1.0, 2.0]).astype(complex)
    nud = np.diag([0.0, 0.0, 0.0, 1.0]).astype(complex)
    pairs = [(-t, c_up.conj().T @ P, c_up), (-t, P @ c_up, c_up.conj().T),
             (-t, c_dn.conj().T @ P, c_dn), (-t, P @ c_dn, c_dn.conj().T)]
    return SparseIMPO([mpohamiltonian(U * nud - mu * n, pairs)])


# ---------------------------------------------------------------------------
# States
# ---------------------------------------------------------------------------
class PeriodicVector(list):
    """1-based periodic list (``PeriodicVector``, ``src/utility.jl:16-53``)."""

    def __getitem__(self, i):
        if isinstance(i, slice):
            return list.__getitem__(self, i)
        return list.__getitem__(self, (i - 1) % len(self))

    def __setitem__(self, i, v):
        list.__setitem__(self, (i - 1) % len(self), v)


def _bond_profile(As):
    return [A.shape[2] for A in As]


class CanonicalIMPS:
    """Device-resident ``CanonicalIMPS`` (``src/states/canonicalmps.jl:17-40``).

    ``AL``, ``AR``, ``C``, ``AC`` download the tensors into 1-based
    ``PeriodicVector``s; ``C[l]`` is the bond right of site ``l`` (``C[0] = C[N]``).
    """

    def __init__(self, ctx: Context, dims: Sequence[int], chi: Sequence[int]):
        self.ctx = ctx
        self.N = len(dims)
        self.dims = list(dims)
        self.chi = list(chi)
        h = C.c_void_p()
        N = self.N
        check(ctx.lib.imps_state_create(ctx.h, N, (C.c_int * N)(*self.dims), (C.c_int * N)(*self.chi), C.byref(h)),
              ctx.h)
        self.h = h
        ctx._adopt(self)

    # constructors -----------------------------------------------------------
    @classmethod
    def from_sites(cls, As: Sequence[np.ndarray], tol=Defaults.tolgauge, maxiter=Defaults.maxiter,
                   ctx: Optional[Context] = None):
        """``CanonicalIMPS(As)``: ``gaugefix!(:LR)`` from ``C0 = I``, ``AC = AL C``."""
        ctx = ctx or default_context()
        N = len(As)
        for l in range(N):
            if As[l].shape[2] != As[(l + 1) % N].shape[0]:
                raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, f"bond mismatch at site {l + 1}")
        psi = cls(ctx, [A.shape[1] for A in As], _bond_profile(As))
        bufs = [cbuf(A) for A in As]
        info = L.GaugeInfo()
        check(ctx.lib.imps_state_canonicalize(psi.h, ptr_array(bufs), tol, maxiter, C.byref(info)), ctx.h)
        psi.gauge_info = info
        return psi

    @classmethod
    def from_AL(cls, ALs: Sequence[np.ndarray], C0: np.ndarray, tol=Defaults.tolgauge, maxiter=Defaults.maxiter,
                ctx: Optional[Context] = None):
        """``CanonicalIMPS(ALs, C0)``: ``gaugefix!(:R)``, ``AC = AL C``."""
        ctx = ctx or default_context()
        N = len(ALs)
        if not (C0.shape[0] == C0.shape[1] == ALs[N - 1].shape[2]):
            raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, "C0 must be chi_N x chi_N")
        psi = cls(ctx, [A.shape[1] for A in ALs], _bond_profile(ALs))
        bufs = [cbuf(A) for A in ALs]
        c0 = cbuf(C0)
        info = L.GaugeInfo()
        check(ctx.lib.imps_state_from_al(psi.h, ptr_array(bufs), dptr(c0), tol, maxiter, C.byref(info)), ctx.h)
        psi.gauge_info = info
        return psi

    def __len__(self):
        return self.N

    def _shape(self, field: int, l: int):
        Dl = self.chi[(l - 1) % self.N]
        Dr = self.chi[l % self.N]
        return (Dr, Dr) if field == L.IMPS_C else (Dl, self.dims[l], Dr)

    def get(self, field: int, l0: int) -> np.ndarray:
        out = np.zeros(self._shape(field, l0), complex, order="F")
        check(self.ctx.lib.imps_state_get(self.h, field, l0, dptr(out)), self.ctx.h)
        return out

    def set(self, field: int, l0: int, a: np.ndarray):
        a = cbuf(a)
        if a.shape != self._shape(field, l0):
            raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, f"expected shape {self._shape(field, l0)}, got {a.shape}")
        check(self.ctx.lib.imps_state_set(self.h, field, l0, dptr(a)), self.ctx.h)

    def _family(self, field):
        return PeriodicVector(self.get(field, l) for l in range(self.N))

    @property
    def AL(self):
        return self._family(L.IMPS_AL)

    @property
    def AR(self):
        return self._family(L.IMPS_AR)

    @property
    def C(self):
        return self._family(L.IMPS_C)

    @property
    def AC(self):
        return self._family(L.IMPS_AC)

    def copy(self):
        out = CanonicalIMPS(self.ctx, self.dims, self.chi)
        check(self.ctx.lib.imps_state_copy(out.h, self.h), self.ctx.h)
        return out

    def dot(self) -> complex:
        """``dot(psi, psi)`` (dominant eigenvalue of the AL transfer matrix)."""
        re, im = C.c_double(), C.c_double()
        check(self.ctx.lib.imps_state_dot(self.h, C.byref(re), C.byref(im)), self.ctx.h)
        return complex(re.value, im.value)

    def norm(self) -> float:
        """``norm(psi) = norm(psi.AC[1])``."""
        return float(np.linalg.norm(self.get(L.IMPS_AC, 0)))

    def _release(self):
        if getattr(self, "h", None):
            self.ctx.lib.imps_state_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass


def random_site_tensors(dims: Sequence[int], D: int, seed: int) -> List[np.ndarray]:
    """Seeded i.i.d. complex-normal ``(D, d, D)`` tensors (Re, Im ~ N(0, 1/2)), NumPy PCG64."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for d in dims:
        re = rng.standard_normal((D, d, D))
        im = rng.standard_normal((D, d, D))
        out.append(np.asfortranarray((re + 1j * im) / math.sqrt(2.0)))
    return out


def randomimps(dims: Sequence[int], D: int, seed: int = 0, ctx: Optional[Context] = None, **kw) -> CanonicalIMPS:
    """``randomimps(ComplexF64, dims; D)`` (``src/states/constructors.jl:13-22``)."""
    if D is None:
        raise ValueError("D must be given explicitly")
    if len(dims) < 1:
        raise ValueError("at least one site is required")
    return CanonicalIMPS.from_sites(random_site_tensors(dims, D, seed), ctx=ctx, **kw)


# ---------------------------------------------------------------------------
# Environments
# ---------------------------------------------------------------------------
class DMRGCache:
    """``DMRGCache(psi, H::SparseIMPO; tol, maxiter, krylovdim)`` on the device."""

    def __init__(self, psi: CanonicalIMPS, H: SparseIMPO, tol=Defaults.tol, maxiter=Defaults.maxiter,
                 krylovdim=Defaults.krylovdim, build=True):
        self.ctx = psi.ctx
        self.operator = H
        h = C.c_void_p()
        check(self.ctx.lib.imps_envs_create(self.ctx.h, psi.h, H.handle(self.ctx), C.byref(h)), self.ctx.h)
        self.h = h
        self.ctx._adopt(self)
        self.N = len(psi)
        self.ml = [H[l + 1].shape[0] for l in range(self.N)]
        self.nr = [H[l + 1].shape[2] for l in range(self.N)]
        self.chi = list(psi.chi)
        self.info = None
        if build:
            self.build(psi, H, tol=tol, maxiter=maxiter, krylovdim=krylovdim, warm=False)

    def build(self, psi, H, tol=Defaults.tol, maxiter=Defaults.maxiter, krylovdim=Defaults.krylovdim, warm=True):
        if isinstance(H, DenseIMPO):
            kinfo = L.KrylovInfo()
            check(self.ctx.lib.imps_envs_build_dense(self.h, psi.h, H.handle(self.ctx), tol, krylovdim, maxiter,
                                                     C.byref(kinfo)), self.ctx.h)
            self.info = kinfo
            return self
        info = L.EnvInfo()
        check(self.ctx.lib.imps_envs_build(self.h, psi.h, H.handle(self.ctx), tol, maxiter, krylovdim, int(warm),
                                           C.byref(info)), self.ctx.h)
        self.info = info
        return self

    def __len__(self):
        return self.N

    def leftenv(self, l: int) -> np.ndarray:
        i = (l - 1) % self.N
        D = self.chi[(i - 1) % self.N]
        out = np.zeros((D, self.ml[i], D), complex, order="F")
        check(self.ctx.lib.imps_envs_get(self.h, 0, i, dptr(out)), self.ctx.h)
        return out

    def rightenv(self, l: int) -> np.ndarray:
        i = (l - 1) % self.N
        D = self.chi[i]
        out = np.zeros((D, self.nr[i], D), complex, order="F")
        check(self.ctx.lib.imps_envs_get(self.h, 1, i, dptr(out)), self.ctx.h)
        return out

    def set_leftenv(self, l: int, GL: np.ndarray):
        check(self.ctx.lib.imps_envs_set(self.h, 0, (l - 1) % self.N, dptr(cbuf(GL))), self.ctx.h)

    def set_rightenv(self, l: int, GR: np.ndarray):
        check(self.ctx.lib.imps_envs_set(self.h, 1, (l - 1) % self.N, dptr(cbuf(GR))), self.ctx.h)

    @property
    def lefts(self):
        return PeriodicVector(self.leftenv(l) for l in range(1, self.N + 1))

    @property
    def rights(self):
        return PeriodicVector(self.rightenv(l) for l in range(1, self.N + 1))

    def _release(self):
        if getattr(self, "h", None):
            self.ctx.lib.imps_envs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass


def recalculate(envs: DMRGCache, psi: CanonicalIMPS, H: Optional[SparseIMPO] = None, tol=Defaults.tol,
                maxiter=Defaults.maxiter, krylovdim=Defaults.krylovdim) -> DMRGCache:
    """``recalculate!(envs, psi, H; tol)``: rebuild in place, warm-started from the old envs."""
    return envs.build(psi, H or envs.operator, tol=tol, maxiter=maxiter, krylovdim=krylovdim, warm=True)


# ---------------------------------------------------------------------------
# Effective Hamiltonians and Krylov calls
# ---------------------------------------------------------------------------
class _ACHam:
    def __init__(self, site, H, envs):
        self.site0 = (site - 1) % envs.N
        self.H = H
        self.envs = envs
        self.shape = (envs.chi[(self.site0 - 1) % envs.N], H[site].shape[1], envs.chi[self.site0])

    def __call__(self, x: np.ndarray) -> np.ndarray:
        x = cbuf(x)
        if x.shape != self.shape:
            raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, f"expected {self.shape}, got {x.shape}")
        y = np.zeros(self.shape, complex, order="F")
        ctx = self.envs.ctx
        check(ctx.lib.imps_ac_apply(self.envs.h, self.H.handle(ctx), self.site0, dptr(x), dptr(y)), ctx.h)
        return y


class _CHam:
    def __init__(self, site, envs):
        self.site0 = (site - 1) % envs.N
        self.envs = envs
        D = envs.chi[self.site0]
        self.shape = (D, D)

    def __call__(self, x: np.ndarray) -> np.ndarray:
        x = cbuf(x)
        if x.shape != self.shape:
            raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, f"expected {self.shape}, got {x.shape}")
        y = np.zeros(self.shape, complex, order="F")
        ctx = self.envs.ctx
        check(ctx.lib.imps_c_apply(self.envs.h, self.site0, dptr(x), dptr(y)), ctx.h)
        return y


def AC_hamiltonian(site: int, below, operator: SparseIMPO, above, envs: DMRGCache) -> _ACHam:
    """``AC_hamiltonian(site, below, operator, above, envs)`` (``effective.jl:66-68``)."""
    return _ACHam(site, operator, envs)


def C_hamiltonian(site: int, below, operator, above, envs: DMRGCache) -> _CHam:
    """``C_hamiltonian(site, ...)`` with ``leftenv(site+1)``, ``rightenv(site)`` (``effective.jl:52-54``)."""
    return _CHam(site, envs)


def fixedpoint(h, x0: np.ndarray, which: str = "SR", alg=None):
    """``fixedpoint(H_AC|H_C, x0, :SR, Lanczos)`` -> ``(lambda, v)`` on the device."""
    if which != "SR":
        raise ValueError("only :SR is supported for the effective Hamiltonians")
    a = _unwrap(alg) if alg is not None else dict(tol=Defaults.tol, krylovdim=30, maxiter=300, eager=True)
    x0 = cbuf(x0)
    x = np.zeros_like(x0)
    info = L.KrylovInfo()
    ctx = h.envs.ctx
    if isinstance(h, _ACHam):
        st = ctx.lib.imps_eigsolve_ac(h.envs.h, h.H.handle(ctx), h.site0, dptr(x0), dptr(x), a["tol"],
                                      a.get("krylovdim", 30), a.get("maxiter", 300), int(a.get("eager", True)),
                                      C.byref(info))
    else:
        st = ctx.lib.imps_eigsolve_c(h.envs.h, h.site0, dptr(x0), dptr(x), a["tol"], a.get("krylovdim", 30),
                                     a.get("maxiter", 300), int(a.get("eager", True)), C.byref(info))
    check(st, ctx.h)
    return info.value_re, x


def integrate(h, x: np.ndarray, dt: complex, alg=None):
    """``integrate(H, x, dt, Lanczos)`` = ``exp(dt H) x`` (``tdvp.jl:14-20``)."""
    a = alg or Defaults.alg_expsolve()
    x0 = cbuf(x)
    out = np.zeros_like(x0)
    info = L.KrylovInfo()
    dt = complex(dt)
    ctx = h.envs.ctx
    if isinstance(h, _ACHam):
        st = ctx.lib.imps_exponentiate_ac(h.envs.h, h.H.handle(ctx), h.site0, dt.real, dt.imag, dptr(x0), dptr(out),
                                          a["tol"], a["krylovdim"], a["maxiter"], C.byref(info))
    else:
        st = ctx.lib.imps_exponentiate_c(h.envs.h, h.site0, dt.real, dt.imag, dptr(x0), dptr(out), a["tol"],
                                         a["krylovdim"], a["maxiter"], C.byref(info))
    check(st, ctx.h)
    return out


def linsolve(dvals: np.ndarray, b: np.ndarray, x0: np.ndarray, a0=1.0, a1=1.0, tol=Defaults.tol,
             krylovdim=Defaults.krylovdim, maxiter=Defaults.maxiter, ctx: Optional[Context] = None):
    """``linsolve`` (GMRES, ``envs.jl:14-19``) for a diagonal operator ``diag(dvals)``."""
    ctx = ctx or default_context()
    d = cbuf(np.ravel(dvals))
    bb = cbuf(np.ravel(b))
    xx = cbuf(np.ravel(x0))
    out = np.zeros_like(bb)
    info = L.KrylovInfo()
    check(ctx.lib.imps_linsolve_diag(ctx.h, bb.size, dptr(d), dptr(bb), dptr(xx), float(a0), float(a1), tol,
                                     krylovdim, maxiter, dptr(out), C.byref(info)), ctx.h)
    return out.reshape(np.shape(b)), info


def qrpos(M: np.ndarray, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    M = cbuf(M)
    m, n = M.shape
    k = min(m, n)
    Q = np.zeros((m, k), complex, order="F")
    R = np.zeros((k, n), complex, order="F")
    check(ctx.lib.imps_qrpos(ctx.h, m, n, dptr(M), dptr(Q), dptr(R)), ctx.h)
    return Q, R


def lqpos(M: np.ndarray, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    M = cbuf(M)
    m, n = M.shape
    k = min(m, n)
    Lf = np.zeros((m, k), complex, order="F")
    Q = np.zeros((k, n), complex, order="F")
    check(ctx.lib.imps_lqpos(ctx.h, m, n, dptr(M), dptr(Lf), dptr(Q)), ctx.h)
    return Lf, Q


def tsvd(M: np.ndarray, kmax: int = 0, cutoff: float = 0.0, ctx: Optional[Context] = None):
    """Truncated SVD ``M = U diag(s) V^H`` on the device (one-sided Jacobi): ``(U, s, V)``
    with ``s`` descending, at most ``kmax`` values (all if 0) above ``cutoff``."""
    ctx = ctx or default_context()
    M = cbuf(M)
    m, n = M.shape
    r = min(m, n)
    U = np.zeros((m, r), complex, order="F")
    V = np.zeros((n, r), complex, order="F")
    s = np.zeros(r)
    k = C.c_int()
    check(ctx.lib.imps_svd(ctx.h, m, n, dptr(M), int(kmax), float(cutoff), dptr(U), s.ctypes.data_as(L.DP),
                           dptr(V), C.byref(k)), ctx.h)
    kk = k.value
    return np.asfortranarray(U[:, :kk]), s[:kk].copy(), np.asfortranarray(V[:, :kk])


def regauge(AC: np.ndarray, Cm: np.ndarray, ctx: Optional[Context] = None) -> np.ndarray:
    """``regauge!(AC, C)`` -> ``AL = Q(AC) Q(C)^H`` (``ortho.jl:214-219``)."""
    ctx = ctx or default_context()
    AC = cbuf(AC)
    Cm = cbuf(Cm)
    Dl, d, Dr = AC.shape
    out = np.zeros_like(AC)
    check(ctx.lib.imps_regauge(ctx.h, Dl, d, Dr, dptr(AC), dptr(Cm), dptr(out)), ctx.h)
    return out


def push_env_left(Lm, above, below=None, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    above = cbuf(above)
    below = above if below is None else cbuf(below)
    Dl, d, Dr = above.shape
    out = np.zeros((Dr, Dr), complex, order="F")
    check(ctx.lib.imps_push_left(ctx.h, Dl, d, Dr, dptr(cbuf(Lm)), dptr(above), dptr(below), dptr(out)), ctx.h)
    return out


def push_env_right(R, above, below=None, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    above = cbuf(above)
    below = above if below is None else cbuf(below)
    Dl, d, Dr = above.shape
    out = np.zeros((Dl, Dl), complex, order="F")
    check(ctx.lib.imps_push_right(ctx.h, Dl, d, Dr, dptr(cbuf(R)), dptr(above), dptr(below), dptr(out)), ctx.h)
    return out


def push_mpo_left(Lm, H: SparseIMPO, site: int, A, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    A = cbuf(A)
    Dl, d, Dr = A.shape
    W = H[site]
    out = np.zeros((Dr, W.shape[2], Dr), complex, order="F")
    check(ctx.lib.imps_push_mpo_left(ctx.h, H.handle(ctx), (site - 1) % len(H), Dl, Dr, dptr(cbuf(Lm)), dptr(A),
                                     dptr(out)), ctx.h)
    return out


def push_mpo_right(R, H: SparseIMPO, site: int, A, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    A = cbuf(A)
    Dl, d, Dr = A.shape
    W = H[site]
    out = np.zeros((Dl, W.shape[0], Dl), complex, order="F")
    check(ctx.lib.imps_push_mpo_right(ctx.h, H.handle(ctx), (site - 1) % len(H), Dl, Dr, dptr(cbuf(R)), dptr(A),
                                      dptr(out)), ctx.h)
    return out


# ---------------------------------------------------------------------------
# Observables
# ---------------------------------------------------------------------------
def calc_galerkin(psi: CanonicalIMPS, H: SparseIMPO, envs: DMRGCache) -> float:
    """``calc_galerkin`` (``vumps.jl:111-124``)."""
    e = C.c_double()
    check(psi.ctx.lib.imps_galerkin(envs.h, H.handle(psi.ctx), psi.h, C.byref(e)), psi.ctx.h)
    return e.value


def expectationvalue(psi: CanonicalIMPS, O=None, envs: Optional[DMRGCache] = None):
    """``expectationvalue(psi, H::SparseIMPO, envs)`` (Schur energy), ``(psi, (i,) => O)``
    local single-site operator, or ``(psi)`` = ``dot(psi, psi)``."""
    ctx = psi.ctx
    if O is None:
        return psi.dot()
    if isinstance(O, DenseIMPO):
        envs = envs or DMRGCache(psi, O)
        re, im = C.c_double(), C.c_double()
        check(ctx.lib.imps_energy_dense(envs.h, O.handle(ctx), psi.h, C.byref(re), C.byref(im)), ctx.h)
        return complex(re.value, im.value)
    if isinstance(O, SparseIMPO):
        envs = envs or DMRGCache(psi, O)
        re, im = C.c_double(), C.c_double()
        check(ctx.lib.imps_energy(envs.h, O.handle(ctx), psi.h, C.byref(re), C.byref(im)), ctx.h)
        return complex(re.value, im.value)
    if isinstance(O, tuple) and len(O) == 2:
        inds, op = O
        sites = tuple(inds) if isinstance(inds, (tuple, list)) else (inds,)
        if len(sites) != 1:
            raise ValueError("only single-site local operators are supported")
        op = cbuf(op)
        re, im = C.c_double(), C.c_double()
        check(ctx.lib.imps_local_expval(psi.h, (sites[0] - 1) % psi.N, dptr(op), C.byref(re), C.byref(im)), ctx.h)
        return complex(re.value, im.value)
    raise TypeError("unsupported operator")


def timeevompo(H: SparseIMPO, delta: complex, alg: str = "WII") -> DenseIMPO:
    """``timeevompo(H::SparseIMPO, delta, WI()/WII())`` (``w1w2.jl:26-31``): the dense MPO
    approximating ``exp(delta H)`` (real time: ``delta = -i dt``; imaginary: ``-tau``), one
    W^I / W^II tensor per site of the unit cell."""
    code = {"WI": 1, "WII": 2}.get(alg)
    if code is None:
        raise L.ArgumentError(L.IMPS_INVALID_ARG, "alg must be 'WI' or 'WII'")
    lib = L.load()
    delta = complex(delta)
    out = []
    for W in H.Ws:
        m, d, n = W.shape[0], W.shape[1], W.shape[2]
        o = np.zeros((m - 1, d, n - 1, d), complex, order="F")
        check(lib.imps_timeevompo_tensor(m, d, n, dptr(cbuf(W)), delta.real, delta.imag, code, dptr(o)))
        out.append(o)
    return DenseIMPO(out)


def dominant_env(psi: CanonicalIMPS, W: Optional[DenseIMPO] = None, side: str = "left", tol=Defaults.tol,
                 krylovdim=Defaults.krylovdim, maxiter=Defaults.maxiter):
    """``dominant_env([W,] psi; side)`` (``envs.jl:34-99``) -> ``(lambda, L)`` with ``L`` of
    shape ``(D, w, D)`` (``w = 1`` without an MPO), unit norm."""
    ctx = psi.ctx
    D = psi.chi[-1]
    w = 1 if W is None else W[1].shape[0]
    L_ = np.zeros((D, w, D), complex, order="F")
    lam = np.zeros(2)
    info = L.KrylovInfo()
    check(ctx.lib.imps_dominant_env(psi.h, None if W is None else W.handle(ctx), 0 if side == "left" else 1, tol,
                                    krylovdim, maxiter, lam.ctypes.data_as(L.DP), dptr(L_), C.byref(info)), ctx.h)
    return complex(lam[0], lam[1]), L_


def correlator(psi: CanonicalIMPS, O1: np.ndarray, O2: np.ndarray, i: int, js) -> np.ndarray:
    """``correlator(psi, O1, O2, i, js)`` (``correlators.jl:13-42``): ``<O1_i O2_j>/<psi|psi>``
    for an int ``js`` (a number) or an increasing range of 1-based sites ``j > i``."""
    single = isinstance(js, (int, np.integer))
    jl = [int(js)] if single else [int(j) for j in js]
    if not jl or jl[0] <= i:
        raise L.ArgumentError(L.IMPS_INVALID_ARG, f"i should be smaller than j ({i}, {jl[0] if jl else None})")
    ctx = psi.ctx
    arr = (C.c_int * len(jl))(*jl)
    out = np.zeros(len(jl), complex)
    check(ctx.lib.imps_correlator(psi.h, dptr(cbuf(O1)), dptr(cbuf(O2)), int(i), len(jl), arr, dptr(out)), ctx.h)
    return out[0] if single else out


def entanglement_spectrum(psi: CanonicalIMPS, loc: int = 1) -> np.ndarray:
    """``entanglement_spectrum(psi, loc)`` (``toolbox.jl:9-14``): normalised squared Schmidt
    values of bond ``loc`` (1-based, right of site ``loc``), descending."""
    b = (loc - 1) % psi.N
    p = np.zeros(psi.chi[b])
    check(psi.ctx.lib.imps_entanglement_spectrum(psi.h, b, p.ctypes.data_as(L.DP)), psi.ctx.h)
    return p


def renyi_entropy(p, alpha: float = 1.0) -> float:
    """von Neumann (``alpha = 1``) or Renyi entropy of a probability vector (natural log)."""
    p = np.asarray(p, dtype=float)
    p = p[p > 0]
    if alpha == 1:
        return float(-np.sum(p * np.log(p)))
    return float(np.log(np.sum(p ** alpha)) / (1.0 - alpha))


def entropy(psi: CanonicalIMPS, loc: int = 1, alpha: float = 1.0) -> float:
    """``entropy(psi, loc; alpha)`` (``toolbox.jl:16-25``)."""
    return renyi_entropy(entanglement_spectrum(psi, loc), alpha)


# ---------------------------------------------------------------------------
# Energy gradients (no counterpart in the reference: an extension for
# gradient-based iMPS optimisation; the right environments are the adjoint
# solution of the left fixed-point system, so nothing iterates)
# ---------------------------------------------------------------------------
def energy_gradient_mpo(psi: CanonicalIMPS, H: SparseIMPO, envs: Optional[DMRGCache] = None) -> List[np.ndarray]:
    """``[dE/dW_1, ..., dE/dW_N]``: derivative of ``expectationvalue(psi, H, envs)``
    with respect to every entry of each site's dense MPO tensor (shape (m, d, n, d)).
    The identity blocks of the Schur form come back as zero."""
    ctx = psi.ctx
    envs = envs or DMRGCache(psi, H)
    out = []
    for l in range(psi.N):
        W = H[l + 1]
        G = np.zeros(W.shape, complex, order="F")
        check(ctx.lib.imps_energy_grad_mpo(envs.h, H.handle(ctx), psi.h, l, dptr(G)), ctx.h)
        out.append(G)
    return out


def energy_gradient_AL(psi: CanonicalIMPS, H: SparseIMPO, envs: Optional[DMRGCache] = None) -> List[np.ndarray]:
    """``[dE/dconj(AL_1), ...]``: Wirtinger gradient of the normalised energy of the
    uniform MPS generated by ``AL``; a direction ``X`` changes E by ``2 Re <g, X>``."""
    ctx = psi.ctx
    envs = envs or DMRGCache(psi, H)
    out = []
    for l in range(psi.N):
        g = np.zeros(psi._shape(L.IMPS_AL, l), complex, order="F")
        check(ctx.lib.imps_energy_grad_al(envs.h, H.handle(ctx), psi.h, l, dptr(g)), ctx.h)
        out.append(g)
    return out


def coupling_gradient(psi: CanonicalIMPS, H: SparseIMPO, dW: Sequence[np.ndarray],
                      envs: Optional[DMRGCache] = None) -> complex:
    """``dE/dtheta`` for an MPO whose site tensors depend on a coupling theta with
    derivatives ``dW[l] = dW_l/dtheta`` (E is linear in each W entry, so this is the
    contraction of ``dW`` with ``energy_gradient_mpo``)."""
    G = energy_gradient_mpo(psi, H, envs)
    return complex(sum(np.sum(np.asarray(dW[l % len(dW)]) * G[l]) for l in range(psi.N)))


def rrule_energy(psi: CanonicalIMPS, H: SparseIMPO, envs: Optional[DMRGCache] = None):
    """Reverse rule for ``expectationvalue(psi, H, envs)``: returns ``(E, pullback)``
    with ``pullback(Ebar) -> (dW list, dAL list)`` (cotangents of the MPO tensors
    and of the conjugated ``AL`` tensors for a real cotangent ``Ebar``)."""
    envs = envs or DMRGCache(psi, H)
    E = expectationvalue(psi, H, envs)
    GW = energy_gradient_mpo(psi, H, envs)
    GA = energy_gradient_AL(psi, H, envs)

    def pullback(Ebar=1.0):
        return [Ebar * g for g in GW], [Ebar * g for g in GA]
    return E, pullback


# ---------------------------------------------------------------------------
# Algorithms
# ---------------------------------------------------------------------------
@dataclass
class VUMPS:
    """``VUMPS(; D, tol, maxiter, verbosity, alg_gauge, alg_eigsolve, alg_environments, finalize)``."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    verbosity: int = Defaults.verbosity
    alg_gauge: object = field(default_factory=Defaults.alg_gauge)
    alg_eigsolve: object = field(default_factory=Defaults.alg_eigsolve)
    alg_environments: object = field(default_factory=Defaults.alg_environments)
    finalize: Optional[Callable] = None


@dataclass
class IDMRG:
    """``IDMRG(; D, tol, maxiter, verbosity, alg_gauge, alg_environments, alg_eigsolve, finalize)``."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    verbosity: int = Defaults.verbosity
    alg_gauge: object = field(default_factory=Defaults.alg_gauge)
    alg_environments: object = field(default_factory=Defaults.alg_environments)
    alg_eigsolve: object = field(default_factory=Defaults.alg_eigsolve)
    finalize: Optional[Callable] = None


@dataclass
class IDMRG2:
    """``IDMRG2(; trunc, tol, maxiter, verbosity, alg_gauge, alg_eigsolve, finalize)``
    (``src/algorithms/algdefs.jl:85-116``) with ``trunc = truncdim(D)``."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    verbosity: int = Defaults.verbosity
    alg_gauge: object = field(default_factory=Defaults.alg_gauge)
    alg_eigsolve: object = field(default_factory=Defaults.alg_eigsolve)
    finalize: Optional[Callable] = None


@dataclass
class VOMPS:
    """``VOMPS(; D, tol, maxiter, verbosity, alg_gauge, alg_environments, alg_orth, finalize)``
    (``src/algorithms/algdefs.jl:118-153``); ``alg_orth`` is QRpos."""
    D: int = Defaults.D
    tol: float = Defaults.tol
    maxiter: int = Defaults.maxiter
    verbosity: int = Defaults.verbosity
    alg_gauge: object = field(default_factory=Defaults.alg_gauge)
    alg_environments: object = field(default_factory=Defaults.alg_environments)
    finalize: Optional[Callable] = None


@dataclass
class TDVP:
    """``TDVP(; integrator, alg_gauge, verbosity, finalize)``."""
    integrator: dict = field(default_factory=Defaults.alg_expsolve)
    alg_gauge: object = field(default_factory=Defaults.alg_gauge)
    verbosity: int = Defaults.verbosity
    finalize: Optional[Callable] = None


@dataclass
class IterativeConvergenceInfo:
    niter: int
    converged: bool
    losses: List[float]
    itererr: float
    residual: Optional[float] = None


def _logiter(name, it, err, **extra):
    s = ", ".join(f"{k} = {v:.8g}" for k, v in extra.items())
    print(f"{name} iter {it:4d} : eps = {err:.3e} {s}")


def find_groundstate(psi0, H: SparseIMPO, alg=None, envs: Optional[DMRGCache] = None, which: str = "SR"):
    """``find_groundstate(psi0, H, alg::VUMPS|IDMRG, [envs])`` -> ``(psi, envs, info)``.

    ``find_groundstate(H, alg)`` (no state) starts from ``randomimps(phydims(H); D = alg.D)``.
    """
    if isinstance(psi0, SparseIMPO):  # convenience form (vumps.jl:96-101)
        H, alg = psi0, H
        psi0 = randomimps(H.phydims(), D=alg.D, seed=0)
    if which != "SR":
        raise ValueError("only :SR is supported")
    if isinstance(alg, IDMRG):
        return _find_groundstate_idmrg(psi0, H, alg, envs)
    if isinstance(alg, IDMRG2):
        return _find_groundstate_idmrg2(psi0, H, alg, envs)
    alg = alg or VUMPS()
    psi = psi0.copy()
    ctx = psi.ctx
    Hh = H.handle(ctx)
    if envs is None:
        envs = DMRGCache(psi0, H)
    eps = calc_galerkin(psi, H, envs)
    ae = updatetol(alg.alg_environments, 0, eps)
    recalculate(envs, psi, H, tol=ae["tol"], maxiter=ae["maxiter"])
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        siter = it - 1
        ea = updatetol(alg.alg_eigsolve, siter, eps)
        nac, nc = C.c_int32(), C.c_int32()
        check(ctx.lib.imps_vumps_localupdate(envs.h, Hh, psi.h, ea["tol"], ea["krylovdim"], ea["maxiter"],
                                             int(ea["eager"]), C.byref(nac), C.byref(nc)), ctx.h)
        ag = updatetol(alg.alg_gauge, siter, eps)
        ginfo = L.GaugeInfo()
        check(ctx.lib.imps_gauge_step(psi.h, ag["tol"], ag["maxiter"], C.byref(ginfo)), ctx.h)
        ae = updatetol(alg.alg_environments, siter, eps)
        recalculate(envs, psi, H, tol=ae["tol"], maxiter=ae["maxiter"])
        if alg.finalize is not None:
            psi, envs = alg.finalize(it, psi, H, envs)
        eps = calc_galerkin(psi, H, envs)
        losses.append(eps)
        if alg.verbosity > 0:
            _logiter("VUMPS", it, eps, f=expectationvalue(psi, H, envs).real)
        if eps <= alg.tol:
            converged = True
            break
    return psi, envs, IterativeConvergenceInfo(it, converged, losses, losses[-1])


def find_groundstate_batch(psi0s: Sequence[CanonicalIMPS], Hs: Sequence[SparseIMPO], alg: Optional[VUMPS] = None,
                           nthreads: int = 16):
    """VUMPS on many independent instances at once -> list of ``(psi, envs, info)``.

    No counterpart in the reference (which would call ``find_groundstate`` per
    instance).  Instances on distinct contexts advance concurrently, one host
    thread and one CUDA stream each (``imps_vumps_iter_batch``); every instance
    follows the default tolerance schedule of ``find_groundstate(::VUMPS)`` and
    stops on its own Galerkin error or ``alg.maxiter``."""
    from concurrent.futures import ThreadPoolExecutor
    alg = alg or VUMPS()
    n = len(psi0s)
    psis = [p.copy() for p in psi0s]

    def setup(i):
        envs = DMRGCache(psis[i], Hs[i])
        eps = calc_galerkin(psis[i], Hs[i], envs)
        ae = updatetol(alg.alg_environments, 0, eps)
        recalculate(envs, psis[i], Hs[i], tol=ae["tol"], maxiter=ae["maxiter"])
        return envs, eps
    # instances sharing a context share its scratch buffers: one host thread per context
    groups = {}
    for i in range(n):
        groups.setdefault(id(psis[i].ctx), []).append(i)
    res = [None] * n

    def setup_group(idx):
        for i in idx:
            res[i] = setup(i)
    with ThreadPoolExecutor(max_workers=max(1, min(nthreads, len(groups)))) as ex:
        list(ex.map(setup_group, groups.values()))
    envss = [r[0] for r in res]
    eps = [r[1] for r in res]
    losses = [[e] for e in eps]
    iters = [0] * n
    converged = [False] * n
    active = [i for i in range(n) if alg.maxiter > 0]
    lib = psis[0].ctx.lib if n else None
    while active:
        k = len(active)
        E = (C.c_void_p * k)(*[envss[i].h for i in active])
        M = (C.c_void_p * k)(*[Hs[i].handle(psis[i].ctx) for i in active])
        S = (C.c_void_p * k)(*[psis[i].h for i in active])
        it = (C.c_int * k)(*[iters[i] + 1 for i in active])
        ep = (C.c_double * k)(*[eps[i] for i in active])
        infos = (L.VumpsInfo * k)()
        st = (C.c_int * k)()
        lib.imps_vumps_iter_batch(k, E, M, S, it, ep, infos, st, nthreads)
        for j, i in enumerate(active):
            check(st[j], psis[i].ctx.h)
            iters[i] += 1
            eps[i] = infos[j].galerkin
            losses[i].append(eps[i])
            converged[i] = eps[i] <= alg.tol
        active = [i for i in active if not converged[i] and iters[i] < alg.maxiter]
    return [(psis[i], envss[i], IterativeConvergenceInfo(iters[i], converged[i], losses[i], losses[i][-1]))
            for i in range(n)]


def _refresh_bonds(psi):
    chi = (C.c_int * psi.N)()
    check(psi.ctx.lib.imps_state_bonds(psi.h, chi), psi.ctx.h)
    psi.chi = list(chi)


def ac2_apply(envs: "DMRGCache", H: SparseIMPO, pos: int, x: np.ndarray) -> np.ndarray:
    """``AC2_hamiltonian(pos, psi, H, psi, envs) * x`` for the window ``(pos, pos+1)``
    (1-based ``pos``, periodic; ``effective.jl:160-197``); ``x`` is ``(Dl, d1, d2, Dr)``."""
    ctx = envs.ctx
    xb = cbuf(x)
    y = np.zeros(xb.shape, complex, order="F")
    check(ctx.lib.imps_ac2_apply(envs.h, H.handle(ctx), (pos - 1) % envs.N, dptr(xb), dptr(y)), ctx.h)
    return y


def _find_groundstate_idmrg2(psi0, H, alg: IDMRG2, envs=None):
    """``find_groundstate(psi0, H, ::IDMRG2)`` (``idmrg.jl:203-235``): two-site sweeps with
    ``truncdim(alg.D)``; the bond dimensions follow the truncation.  Requires N >= 2."""
    if len(psi0) < 2:
        raise L.ArgumentError(L.IMPS_INVALID_ARG, "IDMRG2 requires unit cell length >= 2")
    if isinstance(H, DenseIMPO):
        raise NotImplementedError("IDMRG2 runs on the Schur (SparseIMPO) channel")
    psi = psi0.copy()
    ctx = psi.ctx
    Hh = H.handle(ctx)
    if envs is None:
        envs = DMRGCache(psi0, H)
    eps = calc_galerkin(psi, H, envs)
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        ea = updatetol(alg.alg_eigsolve, it - 1, eps)
        E, err = C.c_double(), C.c_double()
        check(ctx.lib.imps_idmrg2_sweep(envs.h, Hh, psi.h, int(alg.D), ea["tol"], ea["krylovdim"], ea["maxiter"],
                                        int(ea["eager"]), C.byref(E), C.byref(err)), ctx.h)
        _refresh_bonds(psi)
        envs.chi = list(psi.chi)
        if alg.finalize is not None:
            psi, envs = alg.finalize(it, psi, H, envs)
        eps = err.value
        losses.append(eps)
        if alg.verbosity > 0:
            _logiter("IDMRG2", it, eps, f=E.value)
        if eps <= alg.tol:
            converged = True
            break
    ag = updatetol(alg.alg_gauge, it, eps)
    ARs = [psi.get(L.IMPS_AR, l) for l in range(psi.N)]
    psi2 = CanonicalIMPS.from_sites(ARs, tol=ag["tol"], maxiter=ag["maxiter"], ctx=ctx)
    envs2 = DMRGCache(psi2, H, build=False)
    envs2.build(psi2, H, warm=False)
    return psi2, envs2, IterativeConvergenceInfo(it, converged, losses, losses[-1])


class MultCache:
    """``MultCache(bra, W, ket)`` on the device (``src/algorithms/arithmetics/mult.jl:58-197``):
    the ``<bra|W|ket>`` channel's fixed-point environments, ``lefts[l]`` ``(bra, w, ket)`` and
    ``rights[l]`` ``(ket, w, bra)``.  Keeps ``bra``, ``W`` and ``ket`` alive; sweeps change
    ``bra`` in place."""

    def __init__(self, bra: CanonicalIMPS, W: SparseIMPO, ket: CanonicalIMPS, tol=Defaults.tol,
                 maxiter=Defaults.maxiter):
        self.ctx = bra.ctx
        self.bra, self.W, self.ket = bra, W, ket
        self.N = len(bra)
        h = C.c_void_p()
        info = L.KrylovInfo()
        check(self.ctx.lib.imps_mult_envs_create(bra.h, W.handle(self.ctx), ket.h, tol, maxiter, C.byref(h),
                                                 C.byref(info)), self.ctx.h)
        self.h = h
        self.info = info
        self.ctx._adopt(self)

    def _w(self, l):
        return self.W[(l % len(self.W)) + 1]

    def leftenv(self, l: int) -> np.ndarray:
        i = (l - 1) % self.N
        out = np.zeros((self.bra.chi[(i - 1) % self.N], self._w(i).shape[0], self.ket.chi[(i - 1) % self.N]),
                       complex, order="F")
        check(self.ctx.lib.imps_mult_envs_get(self.h, 0, i, dptr(out)), self.ctx.h)
        return out

    def rightenv(self, l: int) -> np.ndarray:
        i = (l - 1) % self.N
        out = np.zeros((self.ket.chi[i], self._w(i).shape[2], self.bra.chi[i]), complex, order="F")
        check(self.ctx.lib.imps_mult_envs_get(self.h, 1, i, dptr(out)), self.ctx.h)
        return out

    def local_maps(self, l: int):
        """``(_local_AC(envs, l), _local_C(envs, l))`` (1-based ``l``)."""
        i = (l - 1) % self.N
        ac = np.zeros(self.bra._shape(L.IMPS_AC, i), complex, order="F")
        c = np.zeros(self.bra._shape(L.IMPS_C, i), complex, order="F")
        check(self.ctx.lib.imps_mult_local_maps(self.h, i, dptr(ac), dptr(c)), self.ctx.h)
        return ac, c

    def galerkin(self) -> float:
        e = C.c_double()
        check(self.ctx.lib.imps_mult_galerkin(self.h, C.byref(e)), self.ctx.h)
        return e.value

    def _release(self):
        if getattr(self, "h", None):
            self.ctx.lib.imps_mult_envs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass


def svdguess_mult(W: SparseIMPO, psi: CanonicalIMPS, D: int, tol=Defaults.tolgauge,
                  maxiter=Defaults.maxiter) -> CanonicalIMPS:
    """``svdguess_mult(W, psi, D)`` (``mult.jl:848-870``): the product ``W psi`` streamed right
    to left through truncating SVDs (bonds <= ``D``), as a mixed-canonical state."""
    ctx = psi.ctx
    h = C.c_void_p()
    info = L.GaugeInfo()
    check(ctx.lib.imps_mult_guess(W.handle(ctx), psi.h, int(D), tol, maxiter, C.byref(h), C.byref(info)), ctx.h)
    out = CanonicalIMPS.__new__(CanonicalIMPS)
    out.ctx = ctx
    out.N = len(psi)
    out.dims = list(psi.dims)
    out.h = h
    ctx._adopt(out)
    _refresh_bonds(out)
    out.gauge_info = info
    return out


def mult(W: SparseIMPO, psi: CanonicalIMPS, alg: Optional[VOMPS] = None):
    """``mult(W, psi, ::VOMPS)`` (``mult.jl:794-806``) -> ``(y, envs, info)``: ``y ~ W psi`` at
    bond dimension ``alg.D``, from ``svdguess_mult`` through ``compression_sweeps!``
    (``arithmetics/envs.jl:51-93``), converged on the Galerkin residual."""
    alg = alg or VOMPS()
    if len(psi) % len(W) != 0:
        raise L.DimensionMismatch(L.IMPS_DIM_MISMATCH, "incompatible unit-cell lengths of MPS and MPO")
    y = svdguess_mult(W, psi, alg.D)
    ae0 = alg.alg_environments.alg if isinstance(alg.alg_environments, DynamicTol) else alg.alg_environments
    envs = MultCache(y, W, psi, tol=ae0["tol"], maxiter=ae0["maxiter"])
    eps = envs.galerkin()
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        ag = updatetol(alg.alg_gauge, it - 1, eps)
        ae = updatetol(alg.alg_environments, it - 1, eps)
        e = C.c_double()
        check(psi.ctx.lib.imps_mult_sweep(envs.h, ag["tol"], ag["maxiter"], ae["tol"], ae["maxiter"], C.byref(e)),
              psi.ctx.h)
        if alg.finalize is not None:
            y, envs = alg.finalize(it, y, W, envs)
        eps = e.value
        losses.append(eps)
        if alg.verbosity > 0:
            _logiter("VOMPS", it, eps)
        if eps <= alg.tol:
            converged = True
            break
    return y, envs, IterativeConvergenceInfo(it, converged, losses, losses[-1])


def _find_groundstate_idmrg(psi0, H, alg: IDMRG, envs=None):
    """``find_groundstate(psi0, H, ::IDMRG)`` (``idmrg.jl:45-82``)."""
    psi = psi0.copy()
    ctx = psi.ctx
    Hh = H.handle(ctx)
    if envs is None:
        envs = DMRGCache(psi0, H)
    eps = calc_galerkin(psi, H, envs)
    losses = [eps]
    converged = False
    it = 0
    for it in range(1, alg.maxiter + 1):
        ea = updatetol(alg.alg_eigsolve, it - 1, eps)
        E, err = C.c_double(), C.c_double()
        check(ctx.lib.imps_idmrg_sweep(envs.h, Hh, psi.h, ea["tol"], ea["krylovdim"], ea["maxiter"],
                                       int(ea["eager"]), C.byref(E), C.byref(err)), ctx.h)
        if alg.finalize is not None:
            psi, envs = alg.finalize(it, psi, H, envs)
        eps = err.value
        losses.append(eps)
        if alg.verbosity > 0:
            _logiter("IDMRG", it, eps, f=E.value)
        if eps <= alg.tol:
            converged = True
            break
    ag = updatetol(alg.alg_gauge, it, eps)
    ARs = [psi.get(L.IMPS_AR, l) for l in range(psi.N)]
    psi2 = CanonicalIMPS.from_sites(ARs, tol=ag["tol"], maxiter=ag["maxiter"], ctx=ctx)
    envs2 = DMRGCache(psi2, H, build=False)
    envs2.build(psi2, H, warm=False)
    return psi2, envs2, IterativeConvergenceInfo(it, converged, losses, losses[-1])


def timestep(psi: CanonicalIMPS, H: SparseIMPO, dt: complex, alg: Optional[TDVP] = None,
             envs: Optional[DMRGCache] = None):
    """``timestep(psi, H, dt, TDVP(), envs)`` -> ``(psi', envs)`` (``tdvp.jl:34-53``)."""
    alg = alg or TDVP()
    psi2 = psi.copy()
    ctx = psi.ctx
    if envs is None:
        envs = DMRGCache(psi2, H)
    g = _unwrap(alg.alg_gauge)
    ig = alg.integrator
    dt = complex(dt)
    info = L.KrylovInfo()
    check(ctx.lib.imps_tdvp_step(envs.h, H.handle(ctx), psi2.h, dt.real, dt.imag, ig["tol"], ig["krylovdim"],
                                 ig["maxiter"], g["tol"], g["maxiter"], C.byref(info)), ctx.h)
    return psi2, envs


def time_evolve(psi0: CanonicalIMPS, H: SparseIMPO, t_span: Sequence[complex], alg: Optional[TDVP] = None,
                envs: Optional[DMRGCache] = None, observer: Optional[Callable] = None):
    """``time_evolve(psi0, H, t_span, alg, envs; observer)`` -> ``(psi, envs, history)``."""
    alg = alg or TDVP()
    psi = psi0.copy()
    if envs is None:
        envs = DMRGCache(psi, H)
    hist = [observer(psi, 0, t_span[0]) if observer else expectationvalue(psi, H, envs)]
    for it in range(1, len(t_span)):
        dt = t_span[it] - t_span[it - 1]
        psi, envs = timestep(psi, H, dt, alg, envs)
        if alg.finalize is not None:
            psi, envs = alg.finalize(t_span[it - 1], psi, H, envs)
        hist.append(observer(psi, it, t_span[it]) if observer else expectationvalue(psi, H, envs))
        if alg.verbosity > 0:
            _logiter("TDVP", it, abs(dt), t=t_span[it])
    return psi, envs, hist
