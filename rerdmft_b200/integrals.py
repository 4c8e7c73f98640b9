"""Two- and three-centre electron-repulsion integrals on the GPU (rr_int_* in include/rr_ri.h), mirroring
the reference's RI set-up functions (src/AO_ints/ThreeCenterIntegrals.h):

* ``auxMetric(aux_basis)``                          ThreeCenterIntegrals.cpp:140-161, (P|Q)
* ``threeCenterIntegralsRaw(basis, aux_basis)``     :163-184, raw[P, p n + q] = (pq|P)
* ``auxMetricOrthogonalization(aux_basis, thr)``    :185-189, canonicalOrthogonalize of the metric
* ``riThreeCenterTensor(basis, aux_basis, metric_x)``  :219-236, B = metric_x^T raw
* ``store_from_basis(basis, aux_basis, ...)``       everything above on the device into a resident
                                                    RiStore (rr_ri_create_basis)

Basis sets are lists of ``basis.BasisFunction`` (as ``basis.build_molecular_basis`` /
``build_auto_auxiliary_basis`` + ``normalize_cartesian_basis`` give them).  ``device=True`` returns CUDA
torch tensors and keeps the result on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from . import basis as bs
from .ri import RiStore, _ptr, canonicalOrthogonalize

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


class _CBasis:
    """An rr_basis over arrays this object keeps alive."""

    def __init__(self, functions):
        self.arrays = bs.flatten(functions)
        a = self.arrays
        self.c = L.Basis(len(functions), a["center"].ctypes.data, a["lxyz"].ctypes.data, a["prim_offset"].ctypes.data,
                         a["exponents"].ctypes.data if a["exponents"].size else None,
                         a["coefficients"].ctypes.data if a["coefficients"].size else None)


def _out(shape, device: bool):
    if device:
        return torch.empty(shape, dtype=torch.float64, device="cuda")
    return np.empty(shape)


def auxMetric(aux_basis, device: bool = False):
    """(P|Q) over the auxiliary functions (naux x naux)."""
    cb = _CBasis(aux_basis)
    n = len(aux_basis)
    M = _out((n, n), device)
    L.check(L.lib().rr_int_aux_metric(ctypes.byref(cb.c), _ptr(M),
                                      ctypes.byref(L.opts(L.RR_MEM_DEVICE if device else L.RR_MEM_HOST))))
    return M


def threeCenterIntegralsRaw(basis, aux_basis, device: bool = False):
    """raw[P, p n + q] = (pq|P), (naux, n^2)."""
    co, ca = _CBasis(basis), _CBasis(aux_basis)
    n, na = len(basis), len(aux_basis)
    raw = _out((na, n * n), device)
    L.check(L.lib().rr_int_three_center_raw(ctypes.byref(co.c), ctypes.byref(ca.c), _ptr(raw),
                                            ctypes.byref(L.opts(L.RR_MEM_DEVICE if device else L.RR_MEM_HOST))))
    return raw


def auxMetricOrthogonalization(aux_basis, threshold: float = 1e-10, report: bool = False):
    """canonicalOrthogonalize of the aux metric: X_metric (naux x naux_kept)."""
    return canonicalOrthogonalize(auxMetric(aux_basis), threshold, report)


def riThreeCenterTensor(basis, aux_basis, metric_x):
    """B = metric_x^T raw (naux_kept, n^2), the integrals and the contraction on the device."""
    from .ri import riThreeCenterTensor as contract

    dev = torch is not None and isinstance(metric_x, torch.Tensor) and metric_x.is_cuda
    return contract(threeCenterIntegralsRaw(basis, aux_basis, device=dev), metric_x)


def store_from_basis(basis, aux_basis, metric_threshold: float = 1e-10, t=None) -> tuple:
    """A resident RiStore from the basis sets, every step on the device (rr_ri_create_basis): the aux
    metric, its canonical orthogonalisation, the raw 3-centre integrals, B = X^T raw and, with t
    (n x n_out), t^T B^P t.  Returns (store, rank report dict)."""
    co, ca = _CBasis(basis), _CBasis(aux_basis)
    tt = np.ascontiguousarray(t, dtype=np.float64) if t is not None else None
    n_out = tt.shape[1] if tt is not None else len(basis)
    st = RiStore.__new__(RiStore)
    st.handle = ctypes.c_void_p()
    kept = ctypes.c_int64(0)
    rep = L.RankReport()
    L.check(L.lib().rr_ri_create_basis(ctypes.byref(co.c), ctypes.byref(ca.c), metric_threshold,
                                       tt.ctypes.data if tt is not None else None, n_out, ctypes.byref(st.handle),
                                       ctypes.byref(kept), ctypes.byref(rep)))
    st.n, st.ns, st.naux = n_out, 0, int(kept.value)
    return st, dict(n_kept=int(rep.n_kept), n_dropped=int(rep.n_dropped), smallest_kept=float(rep.smallest_kept),
                    largest_dropped=float(rep.largest_dropped))
