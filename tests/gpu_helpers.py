"""Helpers shared by the GPU parity tests: move oracle states/environments to the device."""
import numpy as np

import infinitempsalgorithms_b200 as imps
from infinitempsalgorithms_b200 import _lib as L


def upload_state(ctx, opsi):
    """Device CanonicalIMPS holding exactly the oracle state's AL/AR/C/AC."""
    N = len(opsi)
    dims = [a.shape[1] for a in opsi.AL]
    chi = [a.shape[2] for a in opsi.AL]
    psi = imps.CanonicalIMPS(ctx, dims, chi)
    for l in range(N):
        psi.set(L.IMPS_AL, l, opsi.AL[l])
        psi.set(L.IMPS_AR, l, opsi.AR[l])
        psi.set(L.IMPS_C, l, opsi.C[l])
        psi.set(L.IMPS_AC, l, opsi.AC[l])
    return psi


def upload_envs(psi, H, oenvs):
    envs = imps.DMRGCache(psi, H, build=False)
    for l in range(len(psi)):
        envs.set_leftenv(l + 1, oenvs.lefts[l])
        envs.set_rightenv(l + 1, oenvs.rights[l])
    return envs


def to_device_mpo(oH):
    return imps.SparseIMPO(oH.Ws)


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def phase_fix(v, ref):
    ov = np.vdot(ref, v)
    return v * (np.conj(ov) / abs(ov)) if abs(ov) > 0 else v
