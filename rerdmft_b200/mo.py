"""Host-side mirror of the reference's MO-basis RI classes, backed by librr_ri (rr_mo_*).

* ``RiNonRelSpinMoEri`` / ``buildRiNonRelSpinMoEri``   src/NON_REL/NonRelSpinRiMoEri.h:29-102
* ``RiMoEri`` / ``buildRiMoEri``                       src/UKB/RiMoEri.h:30-91
* ``hartreeExchangeFockMatrix`` / ``jkOnlyFockMatrix``  src/Hessian_opt/RiGemmFock.h:20-36

The MO tensor stays resident on the GPU inside the object; ``b()`` copies it out.  ``jkl()``
returns the whole J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i), L_ij = eri(pbar_i,j,j,pbar_i) matrices
the occupation optimiser reads element by element in the reference.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import RrError
from .ri import RiDirectEriSource, RiNonRelEriSource, RiStore, _dev, _host, _is_dev, _ptr


class _MoBase:
    _kind = L.RR_MO_NONREL_SPIN

    def __init__(self, handle: ctypes.c_void_p):
        self.handle = handle
        naux, n, kind = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        L.check(L.lib().rr_mo_info(handle, ctypes.byref(naux), ctypes.byref(n), ctypes.byref(kind)))
        self.naux, self.n = naux.value, n.value

    @classmethod
    def from_tensor(cls, Bmo, n):
        dev = _is_dev(Bmo)
        dt = np.complex128 if cls._kind == L.RR_MO_COMPLEX else np.float64
        B = (_dev if dev else _host)(Bmo, dt)
        h = ctypes.c_void_p()
        L.check(L.lib().rr_mo_from_tensor(_ptr(B), B.shape[0], n, cls._kind, L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST,
                                          ctypes.byref(h)))
        return cls(h)

    def close(self):
        if self.handle and self.handle.value:
            L.lib().rr_mo_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def _dt(self):
        return np.complex128 if self._kind == L.RR_MO_COMPLEX else np.float64

    def dim(self) -> int:
        return self.n if self._kind == L.RR_MO_COMPLEX else 2 * self.n

    dim0 = dim1 = dim2 = dim3 = dim

    def b(self) -> np.ndarray:
        out = np.empty((self.naux, self.n * self.n), dtype=self._dt)
        L.check(L.lib().rr_mo_copy_tensor(self.handle, _ptr(out), ctypes.byref(L.opts())))
        return out

    def eri(self, quads) -> np.ndarray:
        q = np.ascontiguousarray(quads, dtype=np.int64).reshape(-1, 4)
        out = np.empty(q.shape[0], dtype=self._dt)
        L.check(L.lib().rr_mo_eri(self.handle, q.shape[0], _ptr(q), _ptr(out), ctypes.byref(L.opts())))
        return out

    def __call__(self, a, b, c, d):
        return self.eri([[a, b, c, d]])[0]

    def jkl(self, pair_of=None):
        d = self.dim()
        J = np.empty((d, d), dtype=self._dt)
        K = np.empty((d, d), dtype=self._dt)
        Lm = np.empty((d, d), dtype=self._dt) if pair_of is not None else None
        po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
        L.check(L.lib().rr_mo_jkl(self.handle, None if po is None else _ptr(po), _ptr(J), _ptr(K),
                                  None if Lm is None else _ptr(Lm), ctypes.byref(L.opts())))
        return J, K, Lm

    def rotated(self, U):
        dev = _is_dev(U)
        u = (_dev if dev else _host)(U, self._dt)
        h = ctypes.c_void_p()
        o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST)
        L.check(L.lib().rr_mo_rotated(self.handle, _ptr(u), ctypes.byref(h), ctypes.byref(o)))
        return type(self)(h)


class RiNonRelSpinMoEri(_MoBase):
    """src/NON_REL/NonRelSpinRiMoEri.h:29 (real spatial tensor; accessors over 2n spin orbitals)."""

    _kind = L.RR_MO_NONREL_SPIN

    def nSpatial(self) -> int:
        return self.n

    def embeddedB(self) -> np.ndarray:
        out = np.empty((self.naux, 4 * self.n * self.n))
        L.check(L.lib().rr_mo_embedded(self.handle, _ptr(out), ctypes.byref(L.opts())))
        return out


class RiMoEri(_MoBase):
    """src/UKB/RiMoEri.h:30 (complex tensor over n_total spinors)."""

    _kind = L.RR_MO_COMPLEX

    def positiveBlock(self, off: int):
        h = ctypes.c_void_p()
        L.check(L.lib().rr_mo_positive_block(self.handle, off, ctypes.byref(h), ctypes.byref(L.opts())))
        return RiMoEri(h)


def buildRiNonRelSpinMoEri(eri: RiNonRelEriSource | RiStore, n_spatial: int, c_spatial,
                           precision: int = L.RR_PREC_FP64, into: RiNonRelSpinMoEri | None = None) -> RiNonRelSpinMoEri:
    """src/NON_REL/NonRelSpinRiMoEri.cpp:13 on the resident tensor of `eri`.

    precision=RR_PREC_MIXED forms both products in split BF16 on the tensor cores (relative error about
    1e-5 of max|B_mo|); `into` rebuilds an existing tensor of the same shape in place."""
    store = eri.store if isinstance(eri, RiNonRelEriSource) else eri
    if tuple(c_spatial.shape) != (n_spatial, n_spatial):
        raise RrError(L.RR_ERR_ARG, "buildRiNonRelSpinMoEri: c_spatial dimensions do not match n_spatial")
    if store.n != n_spatial:
        raise RrError(L.RR_ERR_ARG, "buildRiNonRelSpinMoEri: eri3_L column count does not match n_spatial*n_spatial")
    dev = _is_dev(c_spatial)
    C = (_dev if dev else _host)(c_spatial, np.float64)
    o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, precision=precision)
    if into is not None:
        L.check(L.lib().rr_mo_build_nonrel_into(store.handle, _ptr(C), into.handle, ctypes.byref(o)))
        return into
    h = ctypes.c_void_p()
    L.check(L.lib().rr_mo_build_nonrel(store.handle, _ptr(C), ctypes.byref(h), ctypes.byref(o)))
    return RiNonRelSpinMoEri(h)


def buildRiMoEri(eri: RiDirectEriSource, c_ukb, precision: int = L.RR_PREC_FP64) -> RiMoEri:
    """src/UKB/RiMoEri.cpp:64 on the resident LL/SS tensors of `eri`.

    precision=RR_PREC_MIXED forms the products in split BF16 on the tensor cores (relative error about
    1e-5 of max|B_mo|)."""
    nu = 2 * eri.nl + 2 * eri.ns
    if c_ukb.shape[0] != nu:
        raise RrError(L.RR_ERR_ARG, "buildRiMoEri: c_ukb row count does not match 2*nLarge+2*nSmall")
    dev = _is_dev(c_ukb)
    c = (_dev if dev else _host)(c_ukb, np.complex128)
    h = ctypes.c_void_p()
    o = L.opts(L.RR_MEM_DEVICE if dev else L.RR_MEM_HOST, precision=precision)
    L.check(L.lib().rr_mo_build_ukb(eri.store.handle, _ptr(c), c.shape[1], ctypes.byref(h), ctypes.byref(o)))
    return RiMoEri(h)


def hartreeExchangeFockMatrix(h, eri: _MoBase, occupations, two_rdm_h, two_rdm_x, pair_of=None, two_rdm_l1=None,
                              two_rdm_l2=None):
    """src/Hessian_opt/RiGemmFock.cpp:161 / :173 (riHxFockGemm) via rr_mo_hx_fock."""
    d = eri.dim()
    if h.shape[0] != d:
        raise RrError(L.RR_ERR_ARG, "hartreeExchangeFockMatrix: eri dimensions inconsistent with h")
    if len(occupations) != d:
        raise RrError(L.RR_ERR_ARG, "hartreeExchangeFockMatrix: occupations size inconsistent with h")
    for m in (two_rdm_h, two_rdm_x):
        if tuple(m.shape) != (d, d):
            raise RrError(L.RR_ERR_ARG, "hartreeExchangeFockMatrix: two_rdm_h/two_rdm_x dimensions inconsistent with h")
    have_l = pair_of is not None and len(pair_of) > 0
    if have_l and (len(pair_of) != d or two_rdm_l1 is None or two_rdm_l2 is None or two_rdm_l1.shape != (d, d)
                   or two_rdm_l2.shape != (d, d)):
        raise RrError(L.RR_ERR_ARG,
                      "hartreeExchangeFockMatrix: pair_of/two_rdm_l1/two_rdm_l2 dimensions inconsistent with h")
    dt = eri._dt
    hh = _host(h, dt)
    args = [_host(occupations, np.float64), _host(two_rdm_h, np.float64), _host(two_rdm_x, np.float64)]
    po = np.ascontiguousarray(pair_of, dtype=np.int64) if have_l else None
    l1 = _host(two_rdm_l1, np.float64) if have_l else None
    l2 = _host(two_rdm_l2, np.float64) if have_l else None
    F = np.empty((d, d), dtype=dt)
    L.check(L.lib().rr_mo_hx_fock(eri.handle, _ptr(hh), *[_ptr(a) for a in args], None if po is None else _ptr(po),
                                  None if l1 is None else _ptr(l1), None if l2 is None else _ptr(l2), _ptr(F),
                                  ctypes.byref(L.opts())))
    return F


def jkOnlyFockMatrix(h, eri: _MoBase, occupations, two_rdm_h, two_rdm_x):
    """src/Hessian_opt/RiGemmFock.cpp:186 / :194: the pair-free special case."""
    return hartreeExchangeFockMatrix(h, eri, occupations, two_rdm_h, two_rdm_x)


# ---------------------------------------------------------------- CASSCF RI operators (src/MCSCF/CasFock.cpp:246-262)


def _dim_dtype(eri):
    return eri.dim(), (np.complex128 if eri._kind == L.RR_MO_COMPLEX else np.float64)


def casTwoElectronOperator(eri, rho):
    """G = J(rho) - K(rho) over the accessor dimension (CasFock.cpp:74-113; embeddedB for the nonrelativistic
    tensor), with K from rho's eigen-decomposition on the device."""
    d, dt = _dim_dtype(eri)
    r = np.ascontiguousarray(rho, dtype=dt)
    if r.shape != (d, d):
        raise RrError(L.RR_ERR_ARG, "casTwoElectronOperator: rho dimension does not match the MO tensor")
    G = np.empty((d, d), dtype=dt)
    L.check(L.lib().rr_mo_cas_two_electron(eri.handle, r.ctypes.data, G.ctypes.data, ctypes.byref(L.opts())))
    return G


def casActiveCumulantFock(eri, active, lam):
    """casActiveCumulantFock (CasFock.cpp:116-133): F (d x a) from the active list and lambda[s,t,r,q]."""
    d, dt = _dim_dtype(eri)
    act = np.ascontiguousarray(active, dtype=np.int64)
    a = act.size
    lm = np.ascontiguousarray(lam, dtype=dt).reshape(-1)
    if lm.size != a ** 4:
        raise RrError(L.RR_ERR_ARG, "casActiveCumulantFock: lambda must hold n_active^4 values")
    F = np.empty((d, a), dtype=dt)
    L.check(L.lib().rr_mo_cas_cumulant_fock(eri.handle, a, act.ctypes.data, lm.ctypes.data, F.ctypes.data,
                                            ctypes.byref(L.opts())))
    return F


def casActiveIntegrals(eri, active):
    """casActiveIntegrals (CasFock.cpp:136-147): (tu|vw) over the active list, a^4 values (flat, [t,u,v,w])."""
    _, dt = _dim_dtype(eri)
    act = np.ascontiguousarray(active, dtype=np.int64)
    out = np.empty(act.size ** 4, dtype=dt)
    L.check(L.lib().rr_mo_cas_active_integrals(eri.handle, act.size, act.ctypes.data, out.ctypes.data,
                                               ctypes.byref(L.opts())))
    return out


def hartreeExchangeJointHessianDiagonal(h, eri, occupations, two_rdm_h, two_rdm_x, fock, pair_indices, pair_of=None,
                                        two_rdm_l1=None, two_rdm_l2=None):
    """hartreeExchangeJointHessianDiagonal on a complex RiMoEri (src/Hessian_opt/HartreeExchangeHessian.cpp:653-711)
    on the GPU: 2 * len(pair_indices) values, the [real; imaginary] diagonal of the joint orbital Hessian.  With
    a PNOF functional's full two-RDM and pair_of this is pnofJointHessianDiagonal (PnofHessian.cpp:171-181)."""
    if eri._kind != L.RR_MO_COMPLEX:
        raise RrError(L.RR_ERR_UNSUPPORTED, "hartreeExchangeJointHessianDiagonal: needs a complex RiMoEri")
    n = eri.n
    hh = np.ascontiguousarray(h, dtype=np.complex128)
    F = np.ascontiguousarray(fock, dtype=np.complex128)
    occ = np.ascontiguousarray(occupations, dtype=np.float64)
    h2 = np.ascontiguousarray(two_rdm_h, dtype=np.float64)
    x2 = np.ascontiguousarray(two_rdm_x, dtype=np.float64)
    if hh.shape != (n, n) or F.shape != (n, n) or occ.size != n or h2.shape != (n, n) or x2.shape != (n, n):
        raise RrError(L.RR_ERR_ARG, "hartreeExchangeJointHessianDiagonal: dimensions inconsistent with the MO tensor")
    pairs = np.ascontiguousarray(pair_indices, dtype=np.int64).reshape(-1, 2)
    po = l1 = l2 = None
    if pair_of is not None:
        po = np.ascontiguousarray(pair_of, dtype=np.int64)
        l1 = np.ascontiguousarray(two_rdm_l1, dtype=np.float64)
        l2 = np.ascontiguousarray(two_rdm_l2, dtype=np.float64)
    out = np.empty(2 * pairs.shape[0])
    L.check(L.lib().rr_mo_hx_joint_hessian_diagonal(
        eri.handle, hh.ctypes.data, occ.ctypes.data, h2.ctypes.data, x2.ctypes.data, F.ctypes.data, pairs.shape[0],
        pairs.ctypes.data if pairs.size else None, None if po is None else po.ctypes.data,
        None if l1 is None else l1.ctypes.data, None if l2 is None else l2.ctypes.data, out.ctypes.data,
        ctypes.byref(L.opts())))
    return out
