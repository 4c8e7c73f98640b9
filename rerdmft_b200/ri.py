"""Host-side mirror of the reference's RI interface, backed by librr_ri (CUDA, sm_100a).

Names, argument meaning and error behaviour follow the reference's C++ overloads:

* ``RiNonRelEriSource`` / ``nonRelFockMatrix``   src/NON_REL/NonRelFockMatrixRi.h:30-40
* ``RiX2cEriSource`` / ``x2cFockMatrix``         src/X2C_DHF/X2C_FockMatrixRi.h:29-40
* ``RiDirectEriSource`` / ``rkbFockMatrix`` / ``riFockTwoElectronDirect``
                                                 src/UKB/UkbFockMatrixRi.h:70-98

The source objects hold the 3-center tensor; here it is uploaded once (lazily, on the first
call) into a resident ``RiStore`` and only the small per-iteration matrices cross to the GPU.
Arguments may be numpy arrays (host; results come back as numpy) or CUDA torch tensors
(device; results stay on the device).  Dimension mismatches raise ``RrError`` (a
``RuntimeError``) with the reference's message, where the reference throws
``std::runtime_error``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import RrError

try:  # torch is only plumbing for device buffers; host (numpy) calls do not need it
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_dev(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _host(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def _dev(a, dtype):
    t = a.contiguous()
    want = torch.float64 if dtype == np.float64 else torch.complex128
    if t.dtype != want:
        t = t.to(want)
    return t


def _ptr(a) -> int:
    if _is_dev(a):
        return a.data_ptr()
    return a.ctypes.data


class RiStore:
    """A resident RI tensor on the current CUDA device (rr_ri_create / rr_ri_create_4c)."""

    def __init__(self, B, B_SS=None, nl=None, ns=None):
        self.handle = ctypes.c_void_p()
        lib = L.lib()
        dev = _is_dev(B)
        conv = _dev if dev else _host
        B = conv(B, np.float64)
        naux = B.shape[0]
        if B_SS is None:
            n = int(round(np.sqrt(B.shape[1]))) if nl is None else nl
            if n * n != B.shape[1]:
                raise RrError(L.RR_ERR_ARG, "RiStore: eri3 column count is not a square")
            L.check(lib.rr_ri_create(_ptr(B), naux, n, L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST,
                                     ctypes.byref(self.handle)))
            self.n, self.ns = n, 0
        else:
            B_SS = conv(B_SS, np.float64)
            if B_SS.shape[0] != naux:
                raise RrError(L.RR_ERR_ARG,
                              "riFockTwoElectronDirect: eri3_LL and eri3_SS do not share the same aux dimension")
            L.check(lib.rr_ri_create_4c(_ptr(B), _ptr(B_SS), naux, nl, ns,
                                        L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, ctypes.byref(self.handle)))
            self.n, self.ns = nl, ns
        self.naux = naux

    def close(self):
        if self.handle and self.handle.value:
            L.lib().rr_ri_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        L.check(L.lib().rr_ri_sync(self.handle))


class RiNonRelEriSource:
    """src/NON_REL/NonRelFockMatrixRi.h:30: nl, eri3_L (n_aux, nl*nl), x_large, overlap.  store: an
    already resident RiStore of the same tensor (e.g. integrals.store_from_basis) in place of eri3_L."""

    def __init__(self, nl, eri3_L, x_large, overlap, store: RiStore | None = None):
        self.nl = int(nl)
        self.eri3_L = eri3_L
        self.x_large = x_large
        self.overlap = overlap
        self._store = store
        if eri3_L is None and (store is None or store.n != self.nl or store.ns != 0):
            raise RrError(L.RR_ERR_ARG, "RiNonRelEriSource: need eri3_L or a single-tensor store of nl functions")

    @property
    def store(self) -> RiStore:
        if self._store is None:
            if self.eri3_L.shape[1] != self.nl * self.nl:
                raise RrError(L.RR_ERR_ARG, "nonRelFockMatrix (RI): eri3_L column count does not match nl^2")
            self._store = RiStore(self.eri3_L, nl=self.nl)
        return self._store


def nonRelFockMatrix(h_core, eri: RiNonRelEriSource, density_matrix, stream: int | None = None):
    """F = h + J - K/2 (src/NON_REL/NonRelFockMatrixRi.cpp:71), computed by rr_ri_fock_nonrel."""
    nl = eri.nl
    if tuple(density_matrix.shape) != (nl, nl):
        raise RrError(L.RR_ERR_ARG, "nonRelFockMatrix (RI): density_matrix dimension does not match nl")
    if eri.eri3_L is not None and eri.eri3_L.shape[1] != nl * nl:
        raise RrError(L.RR_ERR_ARG, "nonRelFockMatrix (RI): eri3_L column count does not match nl^2")
    store = eri.store
    dev = _is_dev(density_matrix)
    conv = _dev if dev else _host
    h = conv(h_core, np.float64)
    D = conv(density_matrix, np.float64)
    S = conv(eri.overlap, np.float64)
    X = conv(eri.x_large, np.float64)
    if tuple(h.shape) != (nl, nl) or tuple(S.shape) != (nl, nl) or X.shape[0] != nl:
        raise RrError(L.RR_ERR_ARG, "nonRelFockMatrix (RI): h_core/overlap/x_large dimensions do not match nl")
    F = torch.empty((nl, nl), dtype=torch.float64, device=D.device) if dev else np.empty((nl, nl))
    o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, stream=stream)
    L.check(L.lib().rr_ri_fock_nonrel(store.handle, _ptr(h), _ptr(D), _ptr(S), _ptr(X), X.shape[1], _ptr(F),
                                      ctypes.byref(o)))
    return F


def jk_occupied(store: RiStore, C_occ, stream: int | None = None):
    """(J, K') for D = 2 C C^T, with F = h + J - K' (rr_ri_jk_occupied)."""
    dev = _is_dev(C_occ)
    conv = _dev if dev else _host
    C = conv(C_occ, np.float64)
    n = store.n
    if C.shape[0] != n:
        raise RrError(L.RR_ERR_ARG, "jk_occupied: C_occ row count does not match n")
    mk = (lambda: torch.empty((n, n), dtype=torch.float64, device=C.device)) if dev else (lambda: np.empty((n, n)))
    J, K = mk(), mk()
    o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, stream=stream)
    L.check(L.lib().rr_ri_jk_occupied(store.handle, _ptr(C), C.shape[1], _ptr(J), _ptr(K), ctypes.byref(o)))
    return J, K


def _cplx_out(shape, like_dev, device=None):
    if like_dev:
        return torch.empty(shape, dtype=torch.complex128, device=device)
    return np.empty(shape, dtype=np.complex128)


class RiX2cEriSource:
    """src/X2C_DHF/X2C_FockMatrixRi.h:29: nl, eri3_L (n_aux, nl*nl) real, x_large / overlap complex."""

    def __init__(self, nl, eri3_L, x_large, overlap):
        self.nl = int(nl)
        self.eri3_L = eri3_L
        self.x_large = x_large
        self.overlap = overlap
        self._store = None

    @property
    def store(self) -> RiStore:
        if self._store is None:
            if self.eri3_L.shape[1] != self.nl * self.nl:
                raise RrError(L.RR_ERR_ARG, "x2cFockMatrix (RI): eri3_L column count does not match nl^2")
            self._store = RiStore(self.eri3_L, nl=self.nl)
        return self._store


def _prec_opts(dev, stream, precision, incremental):
    prec = {"fp64": L.RR_PREC_FP64, "mixed": L.RR_PREC_MIXED}[precision]
    return L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, prec, stream=stream, incremental=1 if incremental else 0)


def x2cFockMatrix(h_x2c, eri: RiX2cEriSource, density_matrix, stream: int | None = None, precision: str = "fp64",
                  incremental: bool = False):
    """src/X2C_DHF/X2C_FockMatrixRi.cpp:79 via rr_ri_fock_x2c (complex 2nl x 2nl).  precision="mixed":
    split-BF16 exchange; incremental=True adds the exchange of the change since the source's previous
    mixed build (a full one when there is none)."""
    n = 2 * eri.nl
    if tuple(density_matrix.shape) != (n, n):
        raise RrError(L.RR_ERR_ARG, "x2cFockMatrix (RI): density_matrix dimension does not match 2*nLarge")
    if eri.eri3_L.shape[1] != eri.nl * eri.nl:
        raise RrError(L.RR_ERR_ARG, "x2cFockMatrix (RI): eri3_L column count does not match nl^2")
    store = eri.store
    dev = _is_dev(density_matrix)
    conv = _dev if dev else _host
    h = conv(h_x2c, np.complex128)
    P = conv(density_matrix, np.complex128)
    S = conv(eri.overlap, np.complex128)
    X = conv(eri.x_large, np.complex128)
    F = _cplx_out((n, n), dev, P.device if dev else None)
    o = _prec_opts(dev, stream, precision, incremental)
    L.check(L.lib().rr_ri_fock_x2c(store.handle, _ptr(h), _ptr(P), _ptr(S), _ptr(X), X.shape[1], _ptr(F),
                                   ctypes.byref(o)))
    return F


class RiDirectEriSource:
    """src/UKB/UkbFockMatrixRi.h:84: nl, ns, eri3_LL, eri3_SS (real), v_total, s_full, x_full (complex)."""

    def __init__(self, nl, ns, eri3_LL, eri3_SS, v_total=None, s_full=None, x_full=None):
        self.nl, self.ns = int(nl), int(ns)
        self.eri3_LL, self.eri3_SS = eri3_LL, eri3_SS
        self.v_total, self.s_full, self.x_full = v_total, s_full, x_full
        self._store = None

    @property
    def store(self) -> RiStore:
        if self._store is None:
            if self.eri3_LL.shape[1] != self.nl ** 2 or self.eri3_SS.shape[1] != self.ns ** 2:
                raise RrError(L.RR_ERR_ARG,
                              "riFockTwoElectronDirect: eri3_LL/eri3_SS column count does not match nl^2/ns^2")
            self._store = RiStore(self.eri3_LL, self.eri3_SS, nl=self.nl, ns=self.ns)
        return self._store


def riFockTwoElectronDirect(eri: RiDirectEriSource, density_ukb, c_occ_ukb, occupations, stream: int | None = None):
    """src/UKB/UkbFockMatrixRi.cpp:35 via rr_ri_two_electron_ukb (the tensors come from `eri`)."""
    nu = 2 * eri.nl + 2 * eri.ns
    if tuple(density_ukb.shape) != (nu, nu):
        raise RrError(L.RR_ERR_ARG, "riFockTwoElectronDirect: density_ukb dimension does not match 2*nLarge+2*nSmall")
    if c_occ_ukb.shape[0] != nu or c_occ_ukb.shape[1] != len(occupations):
        raise RrError(L.RR_ERR_ARG, "riFockTwoElectronDirect: c_occ_ukb dimension does not match n_ukb x occupations.size()")
    store = eri.store
    dev = _is_dev(density_ukb)
    conv = _dev if dev else _host
    P = conv(density_ukb, np.complex128)
    C = conv(c_occ_ukb, np.complex128)
    occ = conv(occupations, np.float64)
    G = _cplx_out((nu, nu), dev, P.device if dev else None)
    o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, stream=stream)
    L.check(L.lib().rr_ri_two_electron_ukb(store.handle, _ptr(P), _ptr(C), C.shape[1], _ptr(occ), _ptr(G),
                                           ctypes.byref(o)))
    return G


def rkbFockMatrix(h_rkb, eri: RiDirectEriSource, density_matrix, stream: int | None = None, precision: str = "fp64",
                  incremental: bool = False):
    """src/UKB/UkbFockMatrixRi.cpp:185 via rr_ri_fock_rkb.  precision / incremental as for x2cFockMatrix."""
    n_rkb = h_rkb.shape[0]
    if tuple(density_matrix.shape) != (n_rkb, n_rkb):
        raise RrError(L.RR_ERR_ARG, "rkbFockMatrix (RI): density_matrix dimension does not match h_rkb")
    store = eri.store
    dev = _is_dev(density_matrix)
    conv = _dev if dev else _host
    h = conv(h_rkb, np.complex128)
    P = conv(density_matrix, np.complex128)
    v = conv(eri.v_total, np.complex128)
    s = conv(eri.s_full, np.complex128)
    x = conv(eri.x_full, np.complex128)
    if v.shape != (2 * eri.nl + 2 * eri.ns, n_rkb) or x.shape[0] != n_rkb:
        raise RrError(L.RR_ERR_ARG, "rkbFockMatrix (RI): v_total/x_full dimensions are inconsistent")
    F = _cplx_out((n_rkb, n_rkb), dev, P.device if dev else None)
    o = _prec_opts(dev, stream, precision, incremental)
    L.check(L.lib().rr_ri_fock_rkb(store.handle, _ptr(h), _ptr(v), n_rkb, _ptr(s), _ptr(x), x.shape[1], _ptr(P),
                                   _ptr(F), ctypes.byref(o)))
    return F


# ---------------------------------------------------------------- one-time set-up on the device


def _setup_call(args_host):
    """Host (numpy) or device (CUDA torch) call of a set-up entry point: all arguments one kind."""
    dev = any(_is_dev(a) for a in args_host if a is not None)
    return dev, L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST)


def _canonical_orth(s, threshold, hermitian, report):
    dev = _is_dev(s)
    dtype = np.complex128 if hermitian else np.float64
    S = _dev(s, dtype) if dev else _host(s, dtype)
    n = S.shape[0]
    if tuple(S.shape) != (n, n):
        raise RrError(L.RR_ERR_ARG, "canonicalOrthogonalize: matrix is not square")
    if dev:
        X = torch.empty(n * n, dtype=torch.complex128 if hermitian else torch.float64, device=S.device)
    else:
        X = np.empty(n * n, dtype=dtype)
    n_eff = ctypes.c_int64(0)
    rep = L.RankReport()
    o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST)
    L.check(L.lib().rr_canonical_orthogonalize(_ptr(S), n, 1 if hermitian else 0, float(threshold), _ptr(X),
                                               ctypes.byref(n_eff), ctypes.byref(rep), ctypes.byref(o)))
    X = X[: n * n_eff.value].reshape(n, n_eff.value)
    if report:
        return X, dict(n_kept=rep.n_kept, n_dropped=rep.n_dropped, smallest_kept=rep.smallest_kept,
                       largest_dropped=rep.largest_dropped)
    return X


def canonicalOrthogonalize(s, threshold: float, report: bool = False):
    """canonicalOrthogonalize (src/Linear_Algebra/LinearAlgebra.cpp:267-310) on the device: X (n x n_eff)
    with X^T S X = I from the eigenvectors of S above `threshold`; the symmetric S^-1/2 when nothing is
    dropped.  report=True also returns the RankReductionReport fields."""
    return _canonical_orth(s, threshold, False, report)


def canonicalOrthogonalizeHermitian(s, threshold: float, report: bool = False):
    """canonicalOrthogonalizeHermitian (LinearAlgebra.cpp:312-349) on the device, with the Jacobi scaling
    D = diag(sqrt(Re S_ii)) applied before the threshold."""
    return _canonical_orth(s, threshold, True, report)


def riThreeCenterTensor(raw, metric_x):
    """riThreeCenterTensor's contraction (src/AO_ints/ThreeCenterIntegrals.cpp:219-236) on the device:
    B = metric_x^T raw for the raw 3-centre integrals (naux_raw, n^2) the host computed."""
    dev, o = _setup_call([raw, metric_x])
    conv = _dev if dev else _host
    raw = conv(raw, np.float64)
    mx = conv(metric_x, np.float64)
    if mx.shape[0] != raw.shape[0]:
        raise RrError(L.RR_ERR_ARG, "riThreeCenterTensor: metric_x row count does not match the raw aux basis size")
    naux_kept, n2 = mx.shape[1], raw.shape[1]
    out = (torch.empty((naux_kept, n2), dtype=torch.float64, device=raw.device) if dev
           else np.empty((naux_kept, n2)))
    L.check(L.lib().rr_ri_three_center_tensor(_ptr(raw), raw.shape[0], n2, _ptr(mx), naux_kept, _ptr(out),
                                              ctypes.byref(o)))
    return out


def transformRiThreeCenterAoLegs(eri3_in, n_ao: int, t):
    """transformRiThreeCenterAoLegs (src/AO_ints/ThreeCenterIntegrals.cpp:191-217) on the device:
    t^T B^P t per aux row."""
    dev, o = _setup_call([eri3_in, t])
    conv = _dev if dev else _host
    B = conv(eri3_in, np.float64)
    t = conv(t, np.float64)
    if B.shape[1] != n_ao * n_ao:
        raise RrError(L.RR_ERR_ARG, "transformRiThreeCenterAoLegs: eri3_in column count does not match n_ao^2")
    if t.shape[0] != n_ao:
        raise RrError(L.RR_ERR_ARG, "transformRiThreeCenterAoLegs: t row count does not match n_ao")
    naux, n_out = B.shape[0], t.shape[1]
    out = (torch.empty((naux, n_out * n_out), dtype=torch.float64, device=B.device) if dev
           else np.empty((naux, n_out * n_out)))
    L.check(L.lib().rr_ri_transform_ao_legs(_ptr(B), naux, n_ao, _ptr(t), n_out, _ptr(out), ctypes.byref(o)))
    return out


def store_from_raw(raw, n_ao: int, metric_x, t=None) -> RiStore:
    """A resident RiStore built on the device from the raw 3-centre integrals (rr_ri_create_raw): the
    metric contraction, then the AO-leg transform when t is given, as the reference builds its source
    tensor (main.cpp:1108 then :4922)."""
    dev = any(_is_dev(a) for a in (raw, metric_x, t) if a is not None)
    conv = _dev if dev else _host
    raw = conv(raw, np.float64)
    mx = conv(metric_x, np.float64)
    if raw.shape[1] != n_ao * n_ao:
        raise RrError(L.RR_ERR_ARG, "riThreeCenterTensor: raw column count does not match n_ao^2")
    if mx.shape[0] != raw.shape[0]:
        raise RrError(L.RR_ERR_ARG, "riThreeCenterTensor: metric_x row count does not match the raw aux basis size")
    tt = conv(t, np.float64) if t is not None else None
    if tt is not None and tt.shape[0] != n_ao:
        raise RrError(L.RR_ERR_ARG, "transformRiThreeCenterAoLegs: t row count does not match n_ao")
    n_out = tt.shape[1] if tt is not None else n_ao
    st = RiStore.__new__(RiStore)
    st.handle = ctypes.c_void_p()
    L.check(L.lib().rr_ri_create_raw(_ptr(raw), raw.shape[0], n_ao, _ptr(mx), mx.shape[1],
                                     _ptr(tt) if tt is not None else None, n_out,
                                     L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, ctypes.byref(st.handle)))
    st.n, st.ns, st.naux = n_out, 0, mx.shape[1]
    return st
