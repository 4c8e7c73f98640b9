"""Device-resident SCF drivers (rr_scf_run_*), mirroring the reference's SCF entry points.

* ``runNonRelativisticHartreeFock``  src/NON_REL/NonRelHartreeFock.cpp:219 (RiNonRelEriSource overload)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .ri import RiNonRelEriSource, _host, _ptr


def _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch, kramers=True):
    prec = {"fp64": L.RR_PREC_FP64, "mixed": L.RR_PREC_MIXED}[precision]
    return L.ScfOpts(diis_size, max_iterations, energy_tolerance, density_tolerance, 1 if kramers else 0, prec,
                     mixed_switch, 0, 0)


def runNonRelativisticHartreeFock(eri: RiNonRelEriSource, h_core, x_large, initial_density, n_electrons: int,
                                  diis_size: int = 5, max_iterations: int = 100, energy_tolerance: float = 1e-8,
                                  density_tolerance: float = 1e-6, precision: str = "fp64",
                                  mixed_switch: float = 1e-5) -> dict:
    """RHF SCF on the GPU; returns energy (electronic), iterations, converged, density P, the
    per-iteration energy history, wall seconds and the mixed / FP64 build counts."""
    n = eri.nl
    h = _host(h_core, np.float64)
    X = _host(x_large, np.float64)
    S = _host(eri.overlap, np.float64)
    P0 = _host(initial_density, np.float64)
    so = _opts(diis_size, max_iterations, energy_tolerance, density_tolerance, precision, mixed_switch)
    res = L.ScfResult()
    P = np.empty((n, n))
    hist = np.full(max_iterations, np.nan)
    L.check(L.lib().rr_scf_run_nonrel(eri.store.handle, _ptr(h), _ptr(X), X.shape[1], _ptr(S), _ptr(P0), n_electrons,
                                      ctypes.byref(so), ctypes.byref(res), _ptr(P), _ptr(hist), ctypes.byref(L.opts())))
    it = int(res.iterations)
    return dict(energy=res.electronic_energy, iterations=it, converged=bool(res.converged), P=P,
                history=hist[:it].copy(), seconds=res.seconds, mixed_iterations=int(res.mixed_iterations),
                fp64_iterations=int(res.fp64_iterations))
