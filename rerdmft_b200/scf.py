"""Device-resident SCF drivers (rr_scf_run_*), mirroring the reference's SCF entry points.

* ``runNonRelativisticHartreeFock``  src/NON_REL/NonRelHartreeFock.cpp:219 (RiNonRelEriSource overload)
* ``runX2CHartreeFockScf``           src/X2C_DHF/X2C_HF.h:131 (RiX2cEriSource overload)
* ``runDiracHartreeFockScf``         src/C4_DHF/C4_DHF.h:116 (RiDirectEriSource overload)

Nuclear repulsion is the caller's (the reference adds it from the geometry); the returned energy
is electronic.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import RrError
from .ri import RiDirectEriSource, RiNonRelEriSource, RiX2cEriSource, _host, _ptr


def _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch, kramers=True,
          mixing=1.0):
    prec = {"fp64": L.RR_PREC_FP64, "mixed": L.RR_PREC_MIXED}[precision]
    return L.ScfOpts(diis_size, max_iterations, energy_tolerance, density_tolerance, 1 if kramers else 0, prec,
                     mixed_switch, mixing)


def _result(res, P, hist, orbitals=None):
    it = int(res.iterations)
    out = dict(energy=res.electronic_energy, iterations=it, converged=bool(res.converged), P=P,
               history=hist[:it].copy(), seconds=res.seconds, mixed_iterations=int(res.mixed_iterations),
               fp64_iterations=int(res.fp64_iterations),
               phase_ms=dict(build=res.build_ms, diis=res.diis_ms, density=res.density_ms))
    if orbitals is not None:
        out.update(orbitals)
    return out


def _request_orbitals(res, n, n_eff, cplx):
    """Host arrays for the loop's optional outputs (the reference's orbital_energies, c_matrix and
    fock_matrix), their pointers set in the result struct."""
    dt = np.complex128 if cplx else np.float64
    o = dict(orbital_energies=np.empty(n_eff), c_matrix=np.empty((n, n_eff), dtype=dt),
             fock_matrix=np.empty((n, n), dtype=dt))
    res.orbital_energies = o["orbital_energies"].ctypes.data
    res.c_matrix = o["c_matrix"].ctypes.data
    res.fock_matrix = o["fock_matrix"].ctypes.data
    return o


def runNonRelativisticHartreeFock(eri: RiNonRelEriSource, h_core, x_large, initial_density, n_electrons: int,
                                  diis_size: int = 5, max_iterations: int = 100, energy_tolerance: float = 1e-8,
                                  density_tolerance: float = 1e-6, precision: str = "fp64",
                                  mixed_switch: float = 0.0, orbitals: bool = False) -> dict:
    """RHF SCF on the GPU; returns energy (electronic), iterations, converged, density P, the
    per-iteration energy history, wall seconds and the mixed / FP64 build counts.  precision="mixed":
    FP64 first build, then incremental split-BF16 exchange, one FP64 build of the final density;
    mixed_switch > 0 re-seeds the accumulated exchange once in FP64 when |dE| < mixed_switch.
    orbitals=True also returns the reference result's orbital_energies, c_matrix and fock_matrix
    (one device diagonalisation of X^T F X at the end of the loop)."""
    n = eri.nl
    h = _host(h_core, np.float64)
    X = _host(x_large, np.float64)
    S = _host(eri.overlap, np.float64)
    P0 = _host(initial_density, np.float64)
    so = _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch)
    res = L.ScfResult()
    orb = _request_orbitals(res, n, X.shape[1], False) if orbitals else None
    P = np.empty((n, n))
    hist = np.full(max_iterations, np.nan)
    L.check(L.lib().rr_scf_run_nonrel(eri.store.handle, _ptr(h), _ptr(X), X.shape[1], _ptr(S), _ptr(P0), n_electrons,
                                      ctypes.byref(so), ctypes.byref(res), _ptr(P), _ptr(hist), ctypes.byref(L.opts())))
    return _result(res, P, hist, orb)


def runX2CHartreeFockScf(h_x2c, eri: RiX2cEriSource, x_large, initial_density, n_electrons: int, overlap=None,
                         diis_size: int = 5, max_iterations: int = 100, energy_tolerance: float = 1e-8,
                         density_tolerance: float = 1e-6, kramers_restricted: bool = True, mixing: float = 1.0,
                         precision: str = "fp64", mixed_switch: float = 0.0, orbitals: bool = False) -> dict:
    """X2C-HF on the GPU (rr_scf_run_x2c).  `overlap` defaults to the source's overlap.
    precision="mixed": incremental split-BF16 exchange, the last iteration an FP64 build of the
    converged density; mixed_switch > 0 re-seeds the accumulated exchange once in FP64 when
    |dE| < mixed_switch.  orbitals as for runNonRelativisticHartreeFock."""
    n = 2 * eri.nl
    S = _host(eri.overlap if overlap is None else overlap, np.complex128)
    h = _host(h_x2c, np.complex128)
    X = _host(x_large, np.complex128)
    P0 = _host(initial_density, np.complex128)
    if h.shape != (n, n) or P0.shape != (n, n) or S.shape != (n, n) or X.shape[0] != n:
        raise RrError(L.RR_ERR_ARG, "runX2CHartreeFockScf: matrix dimensions do not match 2*nLarge")
    so = _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch,
               kramers_restricted, mixing)
    res = L.ScfResult()
    orb = _request_orbitals(res, n, X.shape[1], True) if orbitals else None
    P = np.empty((n, n), dtype=np.complex128)
    hist = np.full(max_iterations, np.nan)
    L.check(L.lib().rr_scf_run_x2c(eri.store.handle, _ptr(h), _ptr(X), X.shape[1], _ptr(S), _ptr(P0), n_electrons,
                                   ctypes.byref(so), ctypes.byref(res), _ptr(P), _ptr(hist), ctypes.byref(L.opts())))
    return _result(res, P, hist, orb)


def runDiracHartreeFockScf(h_rkb, eri: RiDirectEriSource, x_full, initial_density, n_electrons: int, overlap=None,
                           diis_size: int = 5, max_iterations: int = 100, energy_tolerance: float = 1e-8,
                           density_tolerance: float = 1e-6, kramers_restricted: bool = True,
                           mixing: float = 1.0, precision: str = "fp64", mixed_switch: float = 0.0,
                           orbitals: bool = False) -> dict:
    """4c-DHF on the GPU (rr_scf_run_dhf).  `overlap` defaults to the source's s_full.  precision,
    mixed_switch and orbitals as for runX2CHartreeFockScf."""
    h = _host(h_rkb, np.complex128)
    n = h.shape[0]
    S = _host(eri.s_full if overlap is None else overlap, np.complex128)
    X = _host(x_full, np.complex128)
    v = _host(eri.v_total, np.complex128)
    P0 = _host(initial_density, np.complex128)
    if X.shape != (n, n):
        raise RrError(L.RR_ERR_ARG, "rkbDensityMatrix: C_DHF is not square")
    so = _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch,
               kramers_restricted, mixing)
    res = L.ScfResult()
    orb = _request_orbitals(res, n, X.shape[1], True) if orbitals else None
    P = np.empty((n, n), dtype=np.complex128)
    hist = np.full(max_iterations, np.nan)
    L.check(L.lib().rr_scf_run_dhf(eri.store.handle, _ptr(h), _ptr(v), n, _ptr(S), _ptr(X), _ptr(P0), n_electrons,
                                   ctypes.byref(so), ctypes.byref(res), _ptr(P), _ptr(hist), ctypes.byref(L.opts())))
    return _result(res, P, hist, orb)


def runX2CHartreeFockScfBatch(problems, workers: int = 16, diis_size: int = 5, max_iterations: int = 100,
                              energy_tolerance: float = 1e-8, density_tolerance: float = 1e-6,
                              kramers_restricted: bool = True, precision: str = "fp64",
                              mixed_switch: float = 0.0, mode: str = "threads", stats: dict | None = None) -> list:
    """A batch of independent X2C-HF problems (a geometry scan of uneven sizes).  Each problem is a dict
    with eri (RiX2cEriSource), h_x2c, x_large, initial_density, n_electrons and optionally overlap; each
    needs its own handle.  Returns one result dict per problem, as runX2CHartreeFockScf.

    mode "threads": rr_scf_run_x2c_batch, `workers` host threads taking the problems largest store first,
    one stream per problem's handle.  mode "grouped": rr_scf_run_x2c_grouped, all problems in lockstep
    on one stream, every phase of an iteration one grouped launch for all of them (FP64 only); `stats`
    (a dict) receives its launch counts and times."""
    keep, insts = [], (L.X2cInstance * len(problems))()
    outs = []
    for i, pr in enumerate(problems):
        eri = pr["eri"]
        n = 2 * eri.nl
        S = _host(eri.overlap if pr.get("overlap") is None else pr["overlap"], np.complex128)
        h = _host(pr["h_x2c"], np.complex128)
        X = _host(pr["x_large"], np.complex128)
        P0 = _host(pr["initial_density"], np.complex128)
        if h.shape != (n, n) or P0.shape != (n, n) or S.shape != (n, n) or X.shape[0] != n:
            raise RrError(L.RR_ERR_ARG, "runX2CHartreeFockScfBatch: matrix dimensions do not match 2*nLarge")
        P = np.empty((n, n), dtype=np.complex128)
        hist = np.full(max_iterations, np.nan)
        keep += [S, h, X, P0]
        outs.append((P, hist))
        insts[i] = L.X2cInstance(eri.store.handle, _ptr(h), _ptr(X), X.shape[1], _ptr(S), _ptr(P0),
                                 int(pr["n_electrons"]), 0, _ptr(P), _ptr(hist), L.ScfResult())
    so = _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch,
               kramers_restricted, 1.0)
    if mode == "grouped":
        st = L.BatchStats()
        L.check(L.lib().rr_scf_run_x2c_grouped(insts, len(problems), ctypes.byref(so), ctypes.byref(st)))
        if stats is not None:
            stats.update(st.as_dict())
    elif mode == "threads":
        L.check(L.lib().rr_scf_run_x2c_batch(insts, len(problems), ctypes.byref(so), workers))
    else:
        raise RrError(L.RR_ERR_ARG, "runX2CHartreeFockScfBatch: mode is 'threads' or 'grouped'")
    return [_result(insts[i].result, P, hist) for i, (P, hist) in enumerate(outs)]


def autotune_cache(load: str | None = None, save: str | None = None, clear: bool = False) -> int:
    """The grouped GEMM autotuner's cache (rr_autotune_*): optionally clear it, load a cache file, save
    it to a file; returns the number of tuned shapes."""
    if clear:
        L.check(L.lib().rr_autotune_clear())
    if load is not None:
        L.check(L.lib().rr_autotune_load(str(load).encode()))
    if save is not None:
        L.check(L.lib().rr_autotune_save(str(save).encode()))
    return int(L.lib().rr_autotune_entries())
