"""RESTART files (the reference's binary run state, src/Utils/Restart.h) and the hand-over of orbitals
between the runs of a geometry scan, over librr_ri.

* ``RestartData``, ``writeRestart``, ``readRestart``   src/Utils/Restart.h:71-148 (byte-compatible)
* ``restartCoefficients``                              src/Utils/Restart.h:150-153 (C_scf U on the GPU)
* ``densityFromOrbitals``                              the next run's starting density C diag(occ) C^dagger
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class RestartData:
    method: str = "NON_REL"
    functional: str = ""
    kind: str = "OCCUPATIONS"
    basis_fingerprint: int = 0
    n_electrons: int = 0
    pnof_subspaces: int = 0
    pnof_coupling: int = 0
    n_core: int = 0
    jk_frozen_pairs: int = 0
    jk_active_pairs: int = 0
    total_energy: float = 0.0
    orbitals_optimized: bool = False
    converged: bool = False
    occupations: np.ndarray = field(default_factory=lambda: np.zeros(0))
    gammas: np.ndarray = field(default_factory=lambda: np.zeros(0))
    amplitudes: np.ndarray = field(default_factory=lambda: np.zeros(0))
    coefficients: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))  # real or complex, rows x cols
    cas_electrons: int = 0
    cas_spinors: int = 0
    cas_state: np.ndarray = field(default_factory=lambda: np.zeros(0))


def _vec(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return a, (a.ctypes.data if a.size else None), a.size


def writeRestart(path: str, data: RestartData) -> None:
    """writeRestart (src/Utils/Restart.cpp:94-145): the same bytes the reference writes."""
    keep = []
    vecs = {}
    for k in ("occupations", "gammas", "amplitudes", "cas_state"):
        a, p, n = _vec(getattr(data, k))
        keep.append(a)
        vecs[k] = (p, n)
    C = np.asarray(data.coefficients)
    cplx = np.iscomplexobj(C)
    Cc = np.ascontiguousarray(C, dtype=np.complex128 if cplx else np.float64)
    keep.append(Cc)
    rows, cols = (Cc.shape + (0, 0))[:2] if Cc.ndim == 2 else (0, 0)
    r = L.Restart(data.method.encode(), data.functional.encode(), data.kind.encode(), data.basis_fingerprint,
                  data.n_electrons, data.pnof_subspaces, data.pnof_coupling, data.n_core, data.jk_frozen_pairs,
                  data.jk_active_pairs, data.total_energy, 1 if data.orbitals_optimized else 0,
                  1 if data.converged else 0, vecs["occupations"][0], vecs["occupations"][1], vecs["gammas"][0],
                  vecs["gammas"][1], vecs["amplitudes"][0], vecs["amplitudes"][1], 1 if cplx else 0, rows, cols,
                  Cc.ctypes.data if Cc.size else None, data.cas_electrons, data.cas_spinors, vecs["cas_state"][0],
                  vecs["cas_state"][1])
    L.check(L.lib().rr_restart_write(str(path).encode(), ctypes.byref(r)))


def _arr(ptr, n):
    if not ptr or n <= 0:
        return np.zeros(0)
    return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), shape=(n,)).copy()


def readRestart(path: str) -> RestartData:
    """readRestart (src/Utils/Restart.cpp:147-197)."""
    r = L.Restart()
    L.check(L.lib().rr_restart_read(str(path).encode(), ctypes.byref(r)))
    try:
        n = r.rows * r.cols
        if r.complex_coefficients:
            C = _arr(r.coefficients, 2 * n).view(np.complex128).reshape(r.rows, r.cols)
        else:
            C = _arr(r.coefficients, n).reshape(r.rows, r.cols)
        d = RestartData(r.method.decode(), r.functional.decode(), r.kind.decode(), r.basis_fingerprint,
                        r.n_electrons, r.pnof_subspaces, r.pnof_coupling, r.n_core, r.jk_frozen_pairs,
                        r.jk_active_pairs, r.total_energy, bool(r.orbitals_optimized), bool(r.converged),
                        _arr(r.occupations, r.n_occupations), _arr(r.gammas, r.n_gammas),
                        _arr(r.amplitudes, r.n_amplitudes), C, r.cas_electrons, r.cas_spinors,
                        _arr(r.cas_state, r.n_cas_state))
    finally:
        L.lib().rr_restart_release(ctypes.byref(r))
    return d


def restartCoefficients(c_scf, u=None) -> np.ndarray:
    """restartCoefficients (src/Utils/Restart.cpp:199-206): C_scf U on the GPU (U None = identity)."""
    cplx = np.iscomplexobj(c_scf) or (u is not None and np.iscomplexobj(u))
    dt = np.complex128 if cplx else np.float64
    C = np.ascontiguousarray(c_scf, dtype=dt)
    rows, n_mo = C.shape
    if u is not None:
        U = np.ascontiguousarray(u, dtype=dt)
        if U.shape != (n_mo, n_mo):
            raise L.RrError(L.RR_ERR_ARG, "restartCoefficients: rotation size differs from the number of MOs")
    out = np.empty_like(C)
    L.check(L.lib().rr_restart_coefficients(C.ctypes.data, rows, n_mo, None if u is None else U.ctypes.data,
                                            1 if cplx else 0, out.ctypes.data, ctypes.byref(L.opts())))
    return out


def densityFromOrbitals(C, occupations) -> np.ndarray:
    """P = C diag(occ) C^dagger on the GPU: the next run's starting density from a RESTART file's orbitals."""
    cplx = np.iscomplexobj(C)
    Cc = np.ascontiguousarray(C, dtype=np.complex128 if cplx else np.float64)
    occ = np.ascontiguousarray(occupations, dtype=np.float64)
    rows, cols = Cc.shape
    if occ.size != cols:
        raise L.RrError(L.RR_ERR_ARG, "densityFromOrbitals: one occupation per column of C")
    P = np.empty((rows, rows), dtype=Cc.dtype)
    L.check(L.lib().rr_density_from_orbitals(Cc.ctypes.data, rows, cols, occ.ctypes.data, 1 if cplx else 0,
                                             P.ctypes.data, ctypes.byref(L.opts())))
    return P
