"""Test infrastructure only: ctypes access to the reference's OWN RI code.

``oracle/_ref/librrref.so`` is the reference's unmodified RI sources compiled by
``oracle/Makefile`` (see ``ref_bridge.cpp`` for the entry points and the reference
file:line each one calls).  Only tests/, tests/golden/make_golden.py and bench.py's
CPU-baseline leg import this module; the product library never does.

All arrays are row-major numpy float64 / complex128 (interleaved), exactly the
reference's ``Matrix<T>`` layout.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
REF_PATH = _HERE / "_ref" / "librrref.so"
# The same reference objects with the six RI .cpp files replaced by include/rr_ri.hpp over
# librr_ri (`make -C oracle dropin`): the reference's own loops and bridge on the GPU path.
DROPIN_PATH = _HERE / "_ref" / "librrref_dropin.so"
LIB_PATH = DROPIN_PATH if os.environ.get("RRREF_LIB") == "dropin" else REF_PATH
_lib = None

_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_int64)


class ScfResult(ctypes.Structure):
    _fields_ = [("electronic_energy", ctypes.c_double), ("iterations", ctypes.c_int64),
                ("converged", ctypes.c_int64)]


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"reference oracle not built: {LIB_PATH} (run `make -C oracle`)")
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.rrref_last_error.restype = ctypes.c_char_p
        set_threads(int(os.environ.get("RRREF_THREADS", os.cpu_count() or 1)))
    return _lib


def set_threads(n: int) -> None:
    lib_ = _lib if _lib is not None else lib()
    lib_.rrref_set_threads(ctypes.c_int(n))


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    if a.dtype == np.int64:
        return a.ctypes.data_as(_lp)
    return a.ctypes.data_as(_dp)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(lib().rrref_last_error().decode())


def nonrel_fock(h, B, D, S, X):
    n = h.shape[0]
    naux = B.shape[0]
    F = np.empty((n, n))
    B, h, D, S, X = _d(B), _d(h), _d(D), _d(S), _d(X)
    _check(lib().rrref_nonrel_fock(_i64(n), _i64(naux), _p(B), _p(h), _p(D), _p(S), _p(X), _i64(X.shape[1]), _p(F)))
    return F


def x2c_fock(h, B, P, S, X):
    n = h.shape[0]
    nl = n // 2
    F = np.empty((n, n), dtype=np.complex128)
    B, h, P, S, X = _d(B), _c(h), _c(P), _c(S), _c(X)
    _check(lib().rrref_x2c_fock(_i64(nl), _i64(B.shape[0]), _p(B), _p(h), _p(P), _p(S), _p(X), _i64(X.shape[1]),
                                _p(F)))
    return F


def ukb_two_electron(nl, ns, B_LL, B_SS, P_ukb, C_occ, occ):
    nu = 2 * nl + 2 * ns
    G = np.empty((nu, nu), dtype=np.complex128)
    B_LL, B_SS, P_ukb, C_occ, occ = _d(B_LL), _d(B_SS), _c(P_ukb), _c(C_occ), _d(occ)
    _check(lib().rrref_ukb_two_electron(_i64(nl), _i64(ns), _i64(B_LL.shape[0]), _p(B_LL), _p(B_SS), _p(P_ukb),
                                        _p(C_occ), _i64(C_occ.shape[1]), _p(occ), _p(G)))
    return G


def rkb_fock(h, nl, ns, B_LL, B_SS, v_total, s_full, x_full, P):
    n_rkb = h.shape[0]
    F = np.empty((n_rkb, n_rkb), dtype=np.complex128)
    B_LL, B_SS, v_total, s_full, x_full, h, P = _d(B_LL), _d(B_SS), _c(v_total), _c(s_full), _c(x_full), _c(h), _c(P)
    _check(lib().rrref_rkb_fock(_i64(nl), _i64(ns), _i64(B_LL.shape[0]), _p(B_LL), _p(B_SS), _p(v_total),
                                _i64(n_rkb), _p(s_full), _p(x_full), _i64(x_full.shape[1]), _p(h), _p(P), _p(F)))
    return F


def nonrel_mo_build(B, C):
    n = C.shape[0]
    out = np.empty((B.shape[0], n * n))
    B, C = _d(B), _d(C)
    _check(lib().rrref_nonrel_mo_build(_i64(n), _i64(B.shape[0]), _p(B), _p(C), _p(out)))
    return out


def nonrel_mo_rotated(Bmo, n, U):
    out = np.empty_like(Bmo, dtype=np.float64)
    Bmo, U = _d(Bmo), _d(U)
    _check(lib().rrref_nonrel_mo_rotated(_i64(n), _i64(Bmo.shape[0]), _p(Bmo), _p(U), _p(out)))
    return out


def nonrel_mo_embedded(Bmo, n):
    out = np.empty((Bmo.shape[0], 4 * n * n))
    Bmo = _d(Bmo)
    _check(lib().rrref_nonrel_mo_embedded(_i64(n), _i64(Bmo.shape[0]), _p(Bmo), _p(out)))
    return out


def nonrel_mo_eri(Bmo, n, abcd):
    abcd = np.ascontiguousarray(abcd, dtype=np.int64).reshape(-1, 4)
    out = np.empty(abcd.shape[0])
    Bmo = _d(Bmo)
    _check(lib().rrref_nonrel_mo_eri(_i64(n), _i64(Bmo.shape[0]), _p(Bmo), _i64(abcd.shape[0]), _p(abcd), _p(out)))
    return out


def ri_mo_build(nl, ns, B_LL, B_SS, c_ukb):
    n_total = c_ukb.shape[1]
    out = np.empty((B_LL.shape[0], n_total * n_total), dtype=np.complex128)
    B_LL, B_SS, c_ukb = _d(B_LL), _d(B_SS), _c(c_ukb)
    _check(lib().rrref_ri_mo_build(_i64(nl), _i64(ns), _i64(B_LL.shape[0]), _p(B_LL), _p(B_SS), _p(c_ukb),
                                   _i64(n_total), _p(out)))
    return out


def ri_mo_rotated(Bmo, n, U):
    out = np.empty_like(Bmo, dtype=np.complex128)
    Bmo, U = _c(Bmo), _c(U)
    _check(lib().rrref_ri_mo_rotated(_i64(n), _i64(Bmo.shape[0]), _p(Bmo), _p(U), _p(out)))
    return out


def ri_mo_positive(Bmo, n, off):
    m = n - off
    out = np.empty((Bmo.shape[0], m * m), dtype=np.complex128)
    Bmo = _c(Bmo)
    _check(lib().rrref_ri_mo_positive(_i64(n), _i64(Bmo.shape[0]), _p(Bmo), _i64(off), _p(out)))
    return out


def ri_mo_eri(Bmo, n, abcd):
    abcd = np.ascontiguousarray(abcd, dtype=np.int64).reshape(-1, 4)
    out = np.empty(abcd.shape[0], dtype=np.complex128)
    Bmo = _c(Bmo)
    _check(lib().rrref_ri_mo_eri(_i64(n), _i64(Bmo.shape[0]), _p(Bmo), _i64(abcd.shape[0]), _p(abcd), _p(out)))
    return out


def hx_fock_nonrel(Bmo_spatial, n_sp, h, occ, h2, x2, pair_of=None, l1=None, l2=None, use_reference=False):
    n = 2 * n_sp
    F = np.empty((n, n))
    args = [_d(Bmo_spatial), _d(h), _d(occ), _d(h2), _d(x2)]
    po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
    L1 = None if pair_of is None else _d(l1)
    L2 = None if pair_of is None else _d(l2)
    _check(lib().rrref_hx_fock_nonrel(_i64(n_sp), _i64(args[0].shape[0]), *[_p(a) for a in args], _p(po), _p(L1),
                                      _p(L2), ctypes.c_int(1 if use_reference else 0), _p(F)))
    return F


def hx_fock_complex(Bmo, n, h, occ, h2, x2, pair_of=None, l1=None, l2=None, use_reference=False):
    F = np.empty((n, n), dtype=np.complex128)
    args = [_c(Bmo), _c(h), _d(occ), _d(h2), _d(x2)]
    po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
    L1 = None if pair_of is None else _d(l1)
    L2 = None if pair_of is None else _d(l2)
    _check(lib().rrref_hx_fock_complex(_i64(n), _i64(args[0].shape[0]), *[_p(a) for a in args], _p(po), _p(L1),
                                       _p(L2), ctypes.c_int(1 if use_reference else 0), _p(F)))
    return F


def commutator_error(F, P, S):
    n = F.shape[0]
    if np.iscomplexobj(F) or np.iscomplexobj(P) or np.iscomplexobj(S):
        E = np.empty((n, n), dtype=np.complex128)
        _check(lib().rrref_commutator_error_complex(_i64(n), _p(_c(F)), _p(_c(P)), _p(_c(S)), _p(E)))
    else:
        E = np.empty((n, n))
        _check(lib().rrref_commutator_error_real(_i64(n), _p(_d(F)), _p(_d(P)), _p(_d(S)), _p(E)))
    return E


def diis_sequence(max_vectors, errors, values):
    """Feed (errors[t], values[t]) into one reference Diis object; returns (outputs, weight counts)."""
    is_c = np.iscomplexobj(errors) or np.iscomplexobj(values)
    conv = _c if is_c else _d
    errors, values = conv(errors), conv(values)
    steps = errors.shape[0]
    size = errors[0].size
    out = np.empty_like(values)
    wc = np.empty(steps, dtype=np.int64)
    _check(lib().rrref_diis_sequence(ctypes.c_int(1 if is_c else 0), _i64(max_vectors), _i64(steps), _i64(size),
                                     _p(errors), _p(values), _p(out), _p(wc)))
    return out, wc


def canonical_orth(S, thr=1e-10):
    n = S.shape[0]
    n_eff = _i64(0)
    if np.iscomplexobj(S):
        X = np.zeros((n * n,), dtype=np.complex128)
        _check(lib().rrref_canonical_orth_hermitian(_i64(n), _p(_c(S)), ctypes.c_double(thr), _p(X),
                                                    ctypes.byref(n_eff)))
    else:
        X = np.zeros((n * n,))
        _check(lib().rrref_canonical_orth(_i64(n), _p(_d(S)), ctypes.c_double(thr), _p(X), ctypes.byref(n_eff)))
    return X[: n * n_eff.value].reshape(n, n_eff.value)


def _orbital_outputs(n, n_eff, cplx):
    dt = np.complex128 if cplx else np.float64
    return dict(orbital_energies=np.empty(n_eff), c_matrix=np.empty((n, n_eff), dtype=dt),
                fock_matrix=np.empty((n, n), dtype=dt))


def _orb_ptrs(o):
    return _p(o["orbital_energies"]), _p(o["c_matrix"]), _p(o["fock_matrix"])


def canonical_orth_report(S, thr=1e-10):
    """canonicalOrthogonalize{,Hermitian} with its RankReductionReport (n_kept, n_dropped, smallest_kept,
    largest_dropped)."""
    n = S.shape[0]
    herm = np.iscomplexobj(S)
    n_eff = _i64(0)
    X = np.zeros((n * n,), dtype=np.complex128 if herm else np.float64)
    rep = np.zeros(4)
    Sc = _c(S) if herm else _d(S)
    _check(lib().rrref_canonical_orth_report(_i64(n), _p(Sc), ctypes.c_int(1 if herm else 0), ctypes.c_double(thr),
                                             _p(X), ctypes.byref(n_eff), _p(rep)))
    return X[: n * n_eff.value].reshape(n, n_eff.value), dict(n_kept=int(rep[0]), n_dropped=int(rep[1]),
                                                              smallest_kept=rep[2], largest_dropped=rep[3])


def transform_ao_legs(B, n_ao, t):
    """transformRiThreeCenterAoLegs (src/AO_ints/ThreeCenterIntegrals.cpp:191-217): t^T B^P t per aux row."""
    B = _d(B)
    t = _d(t)
    naux, n_out = B.shape[0], t.shape[1]
    out = np.empty((naux, n_out * n_out))
    _check(lib().rrref_transform_ao_legs(_i64(naux), _i64(n_ao), _p(B), _i64(n_out), _p(t), _p(out)))
    return out


def nonrel_scf(sysd, diis_size=5, max_iter=100, e_tol=1e-8, d_tol=1e-6):
    """runNonRelativisticHartreeFock (RI overload): energy, iterations, converged, density, energy history
    and the result's orbital_energies, c_matrix and fock_matrix."""
    n, B = sysd["n"], _d(sysd["B"])
    X = _d(sysd["X"])
    res = ScfResult()
    P = np.empty((n, n))
    hist = np.full(max_iter, np.nan)
    orb = _orbital_outputs(n, X.shape[1], False)
    _check(lib().rrref_nonrel_scf(_i64(n), _i64(B.shape[0]), _p(B), _p(_d(sysd["h"])), _p(X), _i64(X.shape[1]),
                                  _p(_d(sysd["S"])), _p(_d(sysd["D0"])), ctypes.c_int(sysd["n_electrons"]),
                                  ctypes.c_int(diis_size), ctypes.c_int(max_iter), ctypes.c_double(e_tol),
                                  ctypes.c_double(d_tol), ctypes.byref(res), _p(P), _p(hist), *_orb_ptrs(orb)))
    return dict(energy=res.electronic_energy, iterations=res.iterations, converged=bool(res.converged), P=P,
                history=hist[: res.iterations].copy(), **orb)


def x2c_scf(sysd, diis_size=5, max_iter=100, e_tol=1e-8, d_tol=1e-6, kramers=True):
    nl, B = sysd["nl"], _d(sysd["B"])
    X = _c(sysd["X"])
    res = ScfResult()
    P = np.empty((2 * nl, 2 * nl), dtype=np.complex128)
    hist = np.full(max_iter, np.nan)
    orb = _orbital_outputs(2 * nl, X.shape[1], True)
    _check(lib().rrref_x2c_scf(_i64(nl), _i64(B.shape[0]), _p(B), _p(_c(sysd["h"])), _p(X), _i64(X.shape[1]),
                               _p(_c(sysd["S"])), _p(_c(sysd["P0"])), ctypes.c_int(sysd["n_electrons"]),
                               ctypes.c_int(diis_size), ctypes.c_int(max_iter), ctypes.c_double(e_tol),
                               ctypes.c_double(d_tol), ctypes.c_int(1 if kramers else 0), ctypes.byref(res), _p(P),
                               _p(hist), *_orb_ptrs(orb)))
    return dict(energy=res.electronic_energy, iterations=res.iterations, converged=bool(res.converged), P=P,
                history=hist[: res.iterations].copy(), **orb)


def dhf_scf(sysd, diis_size=5, max_iter=100, e_tol=1e-8, d_tol=1e-6, kramers=True):
    nl, ns = sysd["nl"], sysd["ns"]
    n_rkb = sysd["n_rkb"]
    x_full = _c(sysd["x_full"])
    res = ScfResult()
    P = np.empty((n_rkb, n_rkb), dtype=np.complex128)
    hist = np.full(max_iter, np.nan)
    orb = _orbital_outputs(n_rkb, x_full.shape[1], True)
    _check(lib().rrref_dhf_scf(_i64(nl), _i64(ns), _i64(sysd["B_LL"].shape[0]), _p(_d(sysd["B_LL"])),
                               _p(_d(sysd["B_SS"])), _p(_c(sysd["v_total"])), _i64(n_rkb), _p(_c(sysd["s_full"])),
                               _p(x_full), _i64(x_full.shape[1]), _p(_c(sysd["h"])), _p(_c(sysd["P0"])),
                               ctypes.c_int(sysd["n_electrons"]), ctypes.c_int(diis_size), ctypes.c_int(max_iter),
                               ctypes.c_double(e_tol), ctypes.c_double(d_tol), ctypes.c_int(1 if kramers else 0),
                               ctypes.byref(res), _p(P), _p(hist), *_orb_ptrs(orb)))
    return dict(energy=res.electronic_energy, iterations=res.iterations, converged=bool(res.converged), P=P,
                history=hist[: res.iterations].copy(), **orb)


# ---------------------------------------------------------------- orbital-rotation optimisation


def adam_steps(grads, lr=0.01, b1=0.7, b2=0.9, eps=1e-15):
    """Adam<T>::step (src/Utils/ADAM.cpp:33-51) over the rows of `grads` (real or complex)."""
    g = np.ascontiguousarray(grads)
    cplx = np.iscomplexobj(g)
    g = g.astype(np.complex128 if cplx else np.float64)
    out = np.empty_like(g)
    _check(lib().rrref_adam_steps(_i64(g.shape[1]), ctypes.c_int(int(cplx)), _i64(g.shape[0]), ctypes.c_double(lr),
                                  ctypes.c_double(b1), ctypes.c_double(b2), ctypes.c_double(eps),
                                  g.ctypes.data_as(_dp), out.ctypes.data_as(_dp)))
    return out


def adam_run_quadratic(a, b, c, x0, runs):
    """AdamOptimizer<double>::run (ADAM.cpp:140-213) `runs` times on
    E(x) = sum (a x^2/2 + b x) + c (sum x^2)^2 with x += step."""
    a, b, x0 = _d(a), _d(b), _d(x0)
    n = a.size
    eb = np.empty(runs)
    it = np.empty(runs, dtype=np.int32)
    rs = np.empty(runs, dtype=np.int32)
    lr = np.empty(runs)
    x = np.empty(n)
    _check(lib().rrref_adam_run_quadratic(_i64(n), _p(a), _p(b), ctypes.c_double(c), _p(x0), ctypes.c_int(runs),
                                          _p(eb), it.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                          rs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(lr), _p(x)))
    return dict(energy_best=eb, iterations=it, restart=rs.astype(bool), rate=lr, x=x)


def rotation_matrix(kappa):
    """spinorRotationMatrix(kappa) = exp(-kappa) (src/Hessian_opt/SpinorRotation.cpp:17)."""
    k = np.ascontiguousarray(kappa)
    cplx = np.iscomplexobj(k)
    k = k.astype(np.complex128 if cplx else np.float64)
    U = np.empty_like(k)
    _check(lib().rrref_rotation_matrix(_i64(k.shape[0]), ctypes.c_int(int(cplx)), k.ctypes.data_as(_dp),
                                       U.ctypes.data_as(_dp)))
    return U


def orbital_gradient(F):
    """orbitalGradient(F): g_pq = 2 (F_qp - conj F_pq) for p >= q (src/Hessian_opt/OrbitalGradient.h)."""
    f = np.ascontiguousarray(F)
    cplx = np.iscomplexobj(f)
    f = f.astype(np.complex128 if cplx else np.float64)
    g = np.empty_like(f)
    _check(lib().rrref_orbital_gradient(_i64(f.shape[0]), ctypes.c_int(int(cplx)), f.ctypes.data_as(_dp),
                                        g.ctypes.data_as(_dp)))
    return np.tril(g)


def hx_hessian_diag_nonrel(Bmo_spatial, n_sp, h, occ, h2, x2, F, pairs, pair_of=None, l1=None, l2=None):
    """hartreeExchangeHessianElement(p,q,p,q) per pair (src/Hessian_opt/HartreeExchangeHessian.cpp:221)."""
    pr = np.ascontiguousarray(pairs, dtype=np.int64).reshape(-1, 2)
    out = np.empty(pr.shape[0])
    po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
    _check(lib().rrref_hx_hessian_diag_nonrel(_i64(n_sp), _i64(Bmo_spatial.shape[0]), _p(_d(Bmo_spatial)), _p(_d(h)),
                                              _p(_d(occ)), _p(_d(h2)), _p(_d(x2)), _p(_d(F)),
                                              None if po is None else _p(po),
                                              None if po is None else _p(_d(l1)),
                                              None if po is None else _p(_d(l2)), _i64(pr.shape[0]), _p(pr),
                                              _p(out)))
    return out


def hx_energy_nonrel(Bmo_spatial, n_sp, h, occ, h2, x2, pair_of=None, l1=None, l2=None):
    """hartreeExchangeEnergy (src/Hessian_opt/HartreeExchangeGradient.cpp:233)."""
    E = ctypes.c_double()
    po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
    _check(lib().rrref_hx_energy_nonrel(_i64(n_sp), _i64(Bmo_spatial.shape[0]), _p(_d(Bmo_spatial)), _p(_d(h)),
                                        _p(_d(occ)), _p(_d(h2)), _p(_d(x2)), None if po is None else _p(po),
                                        None if po is None else _p(_d(l1)), None if po is None else _p(_d(l2)),
                                        ctypes.byref(E)))
    return E.value


# ---------------------------------------------------------------- RI sigma-vector Hessian-vector primitives
# src/Hessian_opt/RiSigmaGemm.cpp (pairContract, diagContract, accumU) and RiSigmaHessianToolkit.cpp.


def _cplx_of(*arrs):
    return any(a is not None and np.iscomplexobj(a) for a in arrs)


def _cv(a, cplx):
    return None if a is None else (_c(a) if cplx else _d(a))


def sigma_toolkit(B, n, K):
    """buildRiSigmaHessianToolkit(n, B, K): KB1[P] = K B^P, KB2[P] = B^P K and the three diagonals."""
    cplx = np.iscomplexobj(B)
    naux = B.shape[0]
    dt = np.complex128 if cplx else np.float64
    kb1, kb2 = np.empty((naux, n * n), dtype=dt), np.empty((naux, n * n), dtype=dt)
    bd, k1d, k2d = (np.empty((naux, n), dtype=dt) for _ in range(3))
    _check(lib().rrref_sigma_toolkit(_i64(n), _i64(naux), ctypes.c_int(1 if cplx else 0), _p(_cv(B, cplx)),
                                     _p(_d(K)), _p(kb1), _p(kb2), _p(bd), _p(k1d), _p(k2d)))
    return dict(kb1=kb1, kb2=kb2, bdiag=bd, kb1diag=k1d, kb2diag=k2d)


def _op_ptrs(op, cplx):
    s = op.get("s")
    idx = None if s is None else np.ascontiguousarray(op["idx"], dtype=np.uint32)
    keep = [_cv(s, cplx), idx, _cv(op.get("w"), False), _cv(op.get("row"), cplx), _cv(op.get("post"), False)]
    return keep, [None if a is None else _p(a) for a in keep]


def sigma_pair_contract(target, sign, n, naux, f, g):
    """pairContract: target(x,y) + sign sum_{P,t} F(P,t,x) G(P,t,y); an operand is a dict with optional
    s (naux x n^2), idx (n^2 indices into an s row), w (n^2), row (naux x n), post (real n x n)."""
    cplx = _cplx_of(target, f.get("s"), g.get("s"), f.get("row"), g.get("row"))
    out = np.array(target, dtype=np.complex128 if cplx else np.float64, copy=True, order="C")
    kf, pf = _op_ptrs(f, cplx)
    kg, pg = _op_ptrs(g, cplx)
    _check(lib().rrref_sigma_pair_contract(_i64(n), _i64(naux), ctypes.c_int(1 if cplx else 0),
                                           ctypes.c_double(sign), _p(out), *pf, *pg))
    return out


def sigma_diag_contract(target, n, naux, S, Ua=None, Ub=None):
    """diagContract: target(a,b) + sum_P S(P, b n + a) (Ua(P,a) + Ub(P,b))."""
    cplx = _cplx_of(target, S, Ua, Ub)
    out = np.array(target, dtype=np.complex128 if cplx else np.float64, copy=True, order="C")
    ua, ub = _cv(Ua, cplx), _cv(Ub, cplx)
    _check(lib().rrref_sigma_diag_contract(_i64(n), _i64(naux), ctypes.c_int(1 if cplx else 0), _p(out),
                                           _p(_cv(S, cplx)), None if ua is None else _p(ua),
                                           None if ub is None else _p(ub)))
    return out


def sigma_accum_u(U, alpha, n, naux, D, Wm):
    """accumU: U(P,x) + alpha sum_t D[P n + t] Wm(x,t)."""
    cplx = _cplx_of(U, D)
    out = np.array(U, dtype=np.complex128 if cplx else np.float64, copy=True, order="C")
    _check(lib().rrref_sigma_accum_u(_i64(n), _i64(naux), ctypes.c_int(1 if cplx else 0), _p(out),
                                     ctypes.c_double(alpha), _p(_cv(D, cplx)), _p(_d(Wm))))
    return out


# ---------------------------------------------------------------- RESTART files (src/Utils/Restart.cpp)


def restart_write(path, fields):
    """The reference's writeRestart from an rr_restart record (rerdmft_b200._lib.Restart, a plain carrier
    of the same fields)."""
    _check(lib().rrref_restart_write(str(path).encode(), ctypes.byref(fields)))


def restart_rewrite(in_path, out_path):
    """The reference's readRestart of in_path written back with its writeRestart to out_path."""
    _check(lib().rrref_restart_rewrite(str(in_path).encode(), str(out_path).encode()))


# ---------------------------------------------------------------- CASSCF RI operators (src/MCSCF/CasFock.cpp)


def cas_two_electron(Bmo, n, rho):
    """casTwoElectronOperator on RiNonRelSpinMoEri (real Bmo, n spatial orbitals, rho 2n x 2n) or RiMoEri
    (complex Bmo, n spinors)."""
    cplx = np.iscomplexobj(Bmo)
    d = n if cplx else 2 * n
    G = np.empty((d, d), dtype=np.complex128 if cplx else np.float64)
    _check(lib().rrref_cas_two_electron(ctypes.c_int(1 if cplx else 0), _i64(n), _i64(Bmo.shape[0]),
                                        _p(_cv(Bmo, cplx)), _p(_cv(rho, cplx)), _p(G)))
    return G


def cas_cumulant_fock(Bmo, n, active, lam):
    cplx = np.iscomplexobj(Bmo)
    d = n if cplx else 2 * n
    act = np.ascontiguousarray(active, dtype=np.int64)
    F = np.empty((d, act.size), dtype=np.complex128 if cplx else np.float64)
    _check(lib().rrref_cas_cumulant_fock(ctypes.c_int(1 if cplx else 0), _i64(n), _i64(Bmo.shape[0]),
                                         _p(_cv(Bmo, cplx)), _i64(act.size), _p(act),
                                         _p(_cv(np.asarray(lam).reshape(-1), cplx)), _p(F)))
    return F


def cas_active_integrals(Bmo, n, active):
    cplx = np.iscomplexobj(Bmo)
    act = np.ascontiguousarray(active, dtype=np.int64)
    out = np.empty(act.size ** 4, dtype=np.complex128 if cplx else np.float64)
    _check(lib().rrref_cas_active_integrals(ctypes.c_int(1 if cplx else 0), _i64(n), _i64(Bmo.shape[0]),
                                            _p(_cv(Bmo, cplx)), _i64(act.size), _p(act), _p(out)))
    return out


# ---------------------------------------------------------------- joint Hessian diagonal, PNOF two-RDM


def hx_joint_hessian_diag(Bmo, n, h, occ, h2, x2, fock, pairs, pair_of=None, l1=None, l2=None):
    """hartreeExchangeJointHessianDiagonal on a RiMoEri (HartreeExchangeHessian.cpp:653-711)."""
    pr = np.ascontiguousarray(pairs, dtype=np.int64).reshape(-1, 2)
    out = np.empty(2 * pr.shape[0])
    po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
    _check(lib().rrref_hx_joint_hessian_diag(_i64(n), _i64(Bmo.shape[0]), _p(_c(Bmo)), _p(_c(h)), _p(_d(occ)),
                                             _p(_d(h2)), _p(_d(x2)), _p(_c(fock)), _i64(pr.shape[0]), _p(pr),
                                             None if po is None else _p(po), None if l1 is None else _p(_d(l1)),
                                             None if l2 is None else _p(_d(l2)), _p(out)))
    return out


def pnof_full_two_rdm(functional, geminals, occ, n_total, relativistic=True):
    """buildPnofFullTwoRdm + buildPnofPairOf (PnofFock.cpp:29, :139); functional in PNOF5, PNOF7, PNOF7S, GNOF;
    geminals: rows (i, ibar, subspace_id, is_principal)."""
    f = {"PNOF5": 0, "PNOF7": 1, "PNOF7S": 2, "GNOF": 3}[functional]
    g = np.ascontiguousarray(geminals, dtype=np.int64).reshape(-1, 4)
    h2, x2, l1, l2 = (np.empty((n_total, n_total)) for _ in range(4))
    po = np.empty(n_total, dtype=np.int64)
    _check(lib().rrref_pnof_full_two_rdm(ctypes.c_int(f), _i64(g.shape[0]), _p(g), _p(_d(occ)), _i64(n_total),
                                         ctypes.c_int(1 if relativistic else 0), _p(h2), _p(x2), _p(l1), _p(l2),
                                         _p(po)))
    return dict(two_rdm_h=h2, two_rdm_x=x2, two_rdm_l1=l1, two_rdm_l2=l2, pair_of=po)


def pnof_energy_nonrel(functional, geminals, occ, Bmo_spatial, n_sp, h):
    """pnofElectronicEnergy and pnofOccupationGradient (PNOFs.cpp:271, :463) of a non-relativistic
    spin-orbital problem (h and occupations over the 2 n_sp spin orbitals); returns (energy, gradient
    per geminal)."""
    f = {"PNOF5": 0, "PNOF7": 1, "PNOF7S": 2, "GNOF": 3}[functional.upper()]
    g = np.ascontiguousarray(geminals, dtype=np.int64).reshape(-1, 4)
    e = ctypes.c_double()
    grad = np.empty(g.shape[0])
    _check(lib().rrref_pnof_energy_nonrel(ctypes.c_int(f), _i64(g.shape[0]), _p(g), _p(_d(occ)), _i64(n_sp),
                                          _i64(Bmo_spatial.shape[0]), _p(_d(Bmo_spatial)), _p(_d(h)),
                                          ctypes.byref(e), _p(grad)))
    return e.value, grad
