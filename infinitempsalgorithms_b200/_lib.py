"""ctypes binding of ``libimps_b200.so`` (the C ABI in ``include/imps_b200.h``).

The library is built in-tree (``python -m infinitempsalgorithms_b200.build``).
There is no fallback: if the library or a CUDA device is missing, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libimps_b200.so"

IMPS_OK = 0
IMPS_NOT_CONVERGED = 1
IMPS_DIM_MISMATCH = -1
IMPS_INVALID_ARG = -2
IMPS_OOM = -3
IMPS_CUDA_ERROR = -4
IMPS_TIMEOUT = -5
IMPS_NO_DEVICE = -6

IMPS_PREC_FP64 = 0
IMPS_PREC_SPLIT_I8 = 1
IMPS_AL, IMPS_AR, IMPS_C, IMPS_AC = 0, 1, 2, 3


class ImpsError(RuntimeError):
    """A non-OK status from the C ABI."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class DimensionMismatch(ImpsError, ValueError):
    """Mirror of Julia's ``DimensionMismatch`` (reference error behaviour)."""


class ArgumentError(ImpsError, ValueError):
    """Mirror of Julia's ``ArgumentError``."""


class KrylovInfo(C.Structure):
    _fields_ = [("converged", C.c_int32), ("numiter", C.c_int32), ("numops", C.c_int32), ("pad", C.c_int32),
                ("normres", C.c_double), ("value_re", C.c_double), ("value_im", C.c_double)]


class EnvInfo(C.Structure):
    _fields_ = [("solves", C.c_int32), ("gmres_iters", C.c_int32), ("gmres_ops", C.c_int32), ("pushes", C.c_int32),
                ("converged", C.c_int32), ("pad", C.c_int32), ("max_normres", C.c_double)]


class GaugeInfo(C.Structure):
    _fields_ = [("niter", C.c_int32), ("converged", C.c_int32), ("err", C.c_double)]


class VumpsInfo(C.Structure):
    _fields_ = [("galerkin", C.c_double), ("energy_re", C.c_double), ("energy_im", C.c_double),
                ("ac_matvecs", C.c_int32), ("c_matvecs", C.c_int32), ("gauge_iters", C.c_int32),
                ("env_gmres_ops", C.c_int32), ("env", EnvInfo)]


P = C.c_void_p
I32 = C.c_int
I64 = C.c_int64
D = C.c_double
DP = C.POINTER(C.c_double)
PP = C.POINTER(C.c_void_p)

# name -> (restype, argtypes)
_SIGS = {
    "imps_status_string": (C.c_char_p, [I32]),
    "imps_ctx_create": (I32, [I32, PP]),
    "imps_ctx_destroy": (I32, [P]),
    "imps_ctx_set_stream": (I32, [P, P]),
    "imps_ctx_set_precision": (I32, [P, I32, I32]),
    "imps_ctx_synchronize": (I32, [P]),
    "imps_ctx_set_wait_limit": (I32, [P, I64]),
    "imps_timeevompo_tensor": (I32, [I32, I32, I32, DP, D, D, I32, DP]),
    "imps_dominant_env": (I32, [P, P, I32, D, I32, I32, DP, DP, C.POINTER(KrylovInfo)]),
    "imps_envs_build_dense": (I32, [P, P, P, D, I32, I32, C.POINTER(KrylovInfo)]),
    "imps_energy_dense": (I32, [P, P, P, DP, DP]),
    "imps_correlator": (I32, [P, DP, DP, I32, I32, C.POINTER(I32), DP]),
    "imps_entanglement_spectrum": (I32, [P, I32, DP]),
    "imps_svd": (I32, [P, I32, I32, DP, I32, D, DP, DP, DP, C.POINTER(I32)]),
    "imps_ctx_set_workspace_limit": (I32, [P, I64]),
    "imps_ctx_workspace_bytes": (I32, [P, C.POINTER(I64)]),
    "imps_ctx_counters_ext": (I32, [P, C.POINTER(I64), I32]),
    "imps_ctx_last_error": (C.c_char_p, [P]),
    "imps_ctx_profile": (I32, [P, I32]),
    "imps_ctx_profile_get": (I32, [P, C.c_char_p, C.POINTER(I64), DP, DP]),
    "imps_ctx_profile_reset": (I32, [P]),
    "imps_ctx_profile_dump": (I32, [P, C.c_char_p, I64]),
    "imps_ctx_profile_classes": (I32, [P, C.c_char_p]),
    "imps_ctx_counters": (I32, [P, C.POINTER(I64)]),
    "imps_mpo_create": (I32, [P, I32, C.POINTER(I32), C.POINTER(I32), C.POINTER(I32), C.POINTER(DP), PP]),
    "imps_mpo_destroy": (I32, [P]),
    "imps_state_create": (I32, [P, I32, C.POINTER(I32), C.POINTER(I32), PP]),
    "imps_state_destroy": (I32, [P]),
    "imps_state_set": (I32, [P, I32, I32, DP]),
    "imps_state_get": (I32, [P, I32, I32, DP]),
    "imps_state_copy": (I32, [P, P]),
    "imps_state_canonicalize": (I32, [P, C.POINTER(DP), D, I32, C.POINTER(GaugeInfo)]),
    "imps_state_from_al": (I32, [P, C.POINTER(DP), DP, D, I32, C.POINTER(GaugeInfo)]),
    "imps_gauge_step": (I32, [P, D, I32, C.POINTER(GaugeInfo)]),
    "imps_state_dot": (I32, [P, DP, DP]),
    "imps_envs_create": (I32, [P, P, P, PP]),
    "imps_envs_destroy": (I32, [P]),
    "imps_envs_build": (I32, [P, P, P, D, I32, I32, I32, C.POINTER(EnvInfo)]),
    "imps_envs_get": (I32, [P, I32, I32, DP]),
    "imps_envs_set": (I32, [P, I32, I32, DP]),
    "imps_ac_apply": (I32, [P, P, I32, DP, DP]),
    "imps_ac_apply_dev": (I32, [P, P, I32, P, P]),
    "imps_ac_apply_noalloc": (I32, [P, I32, I32, I32, I32, I32, DP, P, P, P, P]),
    "imps_c_apply": (I32, [P, I32, DP, DP]),
    "imps_c_apply_dev": (I32, [P, I32, P, P]),
    "imps_push_left": (I32, [P, I32, I32, I32, DP, DP, DP, DP]),
    "imps_push_right": (I32, [P, I32, I32, I32, DP, DP, DP, DP]),
    "imps_push_mpo_left": (I32, [P, P, I32, I32, I32, DP, DP, DP]),
    "imps_push_mpo_right": (I32, [P, P, I32, I32, I32, DP, DP, DP]),
    "imps_zgemm": (I32, [P, I32, I32, I32, I32, I32, D, D, P, I64, P, I64, D, D, P, I64]),
    "imps_qrpos": (I32, [P, I32, I32, DP, DP, DP]),
    "imps_lqpos": (I32, [P, I32, I32, DP, DP, DP]),
    "imps_regauge": (I32, [P, I32, I32, I32, DP, DP, DP]),
    "imps_eigsolve_ac": (I32, [P, P, I32, DP, DP, D, I32, I32, I32, C.POINTER(KrylovInfo)]),
    "imps_eigsolve_c": (I32, [P, I32, DP, DP, D, I32, I32, I32, C.POINTER(KrylovInfo)]),
    "imps_exponentiate_ac": (I32, [P, P, I32, D, D, DP, DP, D, I32, I32, C.POINTER(KrylovInfo)]),
    "imps_exponentiate_c": (I32, [P, I32, D, D, DP, DP, D, I32, I32, C.POINTER(KrylovInfo)]),
    "imps_linsolve_diag": (I32, [P, I64, DP, DP, DP, D, D, D, I32, I32, DP, C.POINTER(KrylovInfo)]),
    "imps_exponentiate_diag": (I32, [P, I64, DP, D, D, DP, DP, D, I32, I32, C.POINTER(KrylovInfo)]),
    "imps_galerkin": (I32, [P, P, P, DP]),
    "imps_energy": (I32, [P, P, P, DP, DP]),
    "imps_local_expval": (I32, [P, I32, DP, DP, DP]),
    "imps_energy_grad_mpo": (I32, [P, P, P, I32, DP]),
    "imps_energy_grad_al": (I32, [P, P, P, I32, DP]),
    "imps_vumps_localupdate": (I32, [P, P, P, D, I32, I32, I32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "imps_vumps_iter": (I32, [P, P, P, I32, D, C.POINTER(VumpsInfo)]),
    "imps_vumps_iter_batch": (I32, [I32, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(I32), DP,
                                    C.POINTER(VumpsInfo), C.POINTER(I32), I32]),
    "imps_tdvp_step": (I32, [P, P, P, D, D, D, I32, I32, D, I32, C.POINTER(KrylovInfo)]),
    "imps_idmrg_sweep": (I32, [P, P, P, D, I32, I32, I32, DP, DP]),
    "imps_idmrg2_sweep": (I32, [P, P, P, I32, D, I32, I32, I32, DP, DP]),
    "imps_ac2_apply": (I32, [P, P, I32, DP, DP]),
    "imps_state_bonds": (I32, [P, C.POINTER(I32)]),
    "imps_mult_guess": (I32, [P, P, I32, D, I32, PP, C.POINTER(GaugeInfo)]),
    "imps_mult_envs_create": (I32, [P, P, P, D, I32, PP, C.POINTER(KrylovInfo)]),
    "imps_mult_envs_destroy": (I32, [P]),
    "imps_mult_envs_get": (I32, [P, I32, I32, DP]),
    "imps_mult_local_maps": (I32, [P, I32, DP, DP]),
    "imps_mult_galerkin": (I32, [P, DP]),
    "imps_mult_sweep": (I32, [P, D, I32, D, I32, DP]),
}

_lib = None


def load(path: os.PathLike | str | None = None):
    """Load the shared library (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} not found: build it with `python -m infinitempsalgorithms_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


def check(status: int, ctx=None, allow_not_converged: bool = True) -> int:
    if status == IMPS_OK or (status == IMPS_NOT_CONVERGED and allow_not_converged):
        return status
    lib = load()
    msg = lib.imps_ctx_last_error(ctx).decode() if ctx is not None else lib.imps_ctx_last_error(None).decode()
    if status == IMPS_DIM_MISMATCH:
        raise DimensionMismatch(status, msg)
    if status in (IMPS_INVALID_ARG,):
        raise ArgumentError(status, msg)
    raise ImpsError(status, f"{lib.imps_status_string(status).decode()}: {msg}")


def cbuf(a: np.ndarray) -> np.ndarray:
    """Column-major complex128 contiguous copy (the reference's Julia layout)."""
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


def dptr(a: np.ndarray):
    assert a.dtype == np.complex128 and (a.flags.f_contiguous or a.ndim <= 1)
    return a.ctypes.data_as(DP)


def ptr_array(arrs):
    arr = (DP * len(arrs))(*[dptr(a) for a in arrs])
    return arr
