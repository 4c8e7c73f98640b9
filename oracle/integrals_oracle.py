"""CPU restatement of the reference's Gaussian integrals (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this module, and only
as the checker; the product path (``rerdmft_b200.integrals`` + ``librr_ri.so``) never calls it.

The reference takes every integral from libcint 5.1.6 (third-party, un-vendored, absent here):
``cint1e_ovlp_cart`` (src/AO_ints/Integrals.cpp:64-129), kinetic and nuclear attraction
(src/AO_ints/SchrodingerKinetic.cpp, NuclearAttraction.cpp), ``cint2c2e_cart`` and ``cint3c2e_cart``
(src/AO_ints/ThreeCenterIntegrals.cpp:25-138).  The integrals are defined by the mathematics, so this
module restates them with McMurchie and Davidson's Hermite-Gaussian scheme (J. Comput. Phys. 26, 218
(1978); the recurrences as in Helgaker, Jorgensen, Olsen, "Molecular Electronic-Structure Theory",
ch. 9), with libcint's conventions for what a coefficient multiplies: coefficient * f(l) *
x^lx y^ly z^lz exp(-a r^2), f(0) = 1/sqrt(4 pi), f(1) = sqrt(3/(4 pi)), f(l >= 2) = 1 (the reference
states this at src/Utils/AIMPAC.cpp:100-106).  The Boys function comes from scipy's regularised
incomplete gamma function, independent of the device code's own evaluation.

Pins (tests/test_integrals_oracle.py): the Boys function against its series, s-type integrals against
their closed forms, p and d functions against finite differences of s functions in the centre
coordinates, and the RI Hartree-Fock energy of LiH / 6-31G built from these integrals against the
reference's own printed value (examples/reference.yaml, fixture tests/golden/lih_631g.npz).

Layouts: ``aux_metric`` -> (naux, naux); ``three_center_raw`` -> (naux, n*n) with raw[P, p*n + q] = (pq|P)
(src/AO_ints/ThreeCenterIntegrals.cpp:163-184).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import gamma as _gamma
from scipy.special import gammainc as _gammainc


def _common(l: int) -> float:
    return 1.0 / math.sqrt(4.0 * math.pi) if l == 0 else (math.sqrt(3.0 / (4.0 * math.pi)) if l == 1 else 1.0)


def _components(l: int):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def boys(nmax: int, T) -> np.ndarray:
    """F_n(T) = int_0^1 t^(2n) exp(-T t^2) dt for n = 0..nmax: (nmax+1,) + T.shape.
    F_n(T) = gamma(n + 1/2) P(n + 1/2, T) / (2 T^(n + 1/2)), P the regularised lower incomplete gamma;
    below T = 1e-8 the first terms of the Taylor series."""
    T = np.asarray(T, dtype=np.float64)
    out = np.empty((nmax + 1,) + T.shape)
    small = T < 1e-8
    Ts = np.where(small, 1.0, T)
    for n in range(nmax + 1):
        big = _gamma(n + 0.5) * _gammainc(n + 0.5, Ts) / (2.0 * Ts ** (n + 0.5))
        ser = 1.0 / (2 * n + 1) - T / (2 * n + 3) + T * T / (2.0 * (2 * n + 5))
        out[n] = np.where(small, ser, big)
    return out


def hermite_e(la: int, lb: int, a, b, xab):
    """E[i][j][t] (i <= la, j <= lb, t <= i + j) of the 1-D overlap distribution of x_A^i x_B^j exp(-a x_A^2 -
    b x_B^2), without the exp(-ab/p X_AB^2) factor; broadcast over the shapes of a, b, xab."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    p = a + b
    xpa = -b / p * xab
    xpb = a / p * xab
    shape = np.broadcast(a, b, np.asarray(xab)).shape
    zero = np.zeros(shape)
    E = [[[zero for _ in range(la + lb + 2)] for _ in range(lb + 1)] for _ in range(la + 1)]
    E[0][0][0] = np.ones(shape)
    inv2p = 0.5 / p
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            for t in range(i + j + 1):
                if i > 0:
                    src, x = E[i - 1][j], xpa
                else:
                    src, x = E[i][j - 1], xpb
                v = x * src[t]
                if t > 0:
                    v = v + inv2p * src[t - 1]
                if t + 1 < len(src):
                    v = v + (t + 1) * src[t + 1]
                E[i][j][t] = v
    return E


def hermite_r(L: int, alpha, X, Y, Z) -> dict:
    """R_{tuv}(alpha, R_PC) for t + u + v <= L (Hermite Coulomb integrals), {(t, u, v): array}."""
    alpha = np.asarray(alpha, dtype=np.float64)
    T = alpha * (X * X + Y * Y + Z * Z)
    F = boys(L, T)
    cur = {}
    for n in range(L, -1, -1):
        nxt = {(0, 0, 0): (-2.0 * alpha) ** n * F[n]}
        for s in range(1, L - n + 1):
            for t in range(s, -1, -1):
                for u in range(s - t, -1, -1):
                    v = s - t - u
                    if t > 0:
                        val = X * cur[(t - 1, u, v)]
                        if t > 1:
                            val = val + (t - 1) * cur[(t - 2, u, v)]
                    elif u > 0:
                        val = Y * cur[(t, u - 1, v)]
                        if u > 1:
                            val = val + (u - 1) * cur[(t, u - 2, v)]
                    else:
                        val = Z * cur[(t, u, v - 1)]
                        if v > 1:
                            val = val + (v - 1) * cur[(t, u, v - 2)]
                    nxt[(t, u, v)] = val
        cur = nxt
    return cur


class _Sh:
    """A contracted shell: centre, l, exponents, coefficients (the libcint-convention coefficients of its
    representative function) and per-component scales relative to it."""

    def __init__(self, center, l, exps, coefs):
        self.c = np.asarray(center, dtype=np.float64)
        self.l = int(l)
        self.a = np.asarray(exps, dtype=np.float64)
        self.k = np.asarray(coefs, dtype=np.float64) * _common(self.l)


def _shell_of(fn) -> _Sh:
    return _Sh((fn.x, fn.y, fn.z), fn.l, fn.exponents, fn.coefficients)


def _shell_blocks(basis):
    """[(shell, [(component index, function index, scale)])]: consecutive components sharing centre, l,
    exponents and proportional coefficients form one shell; any other function is a shell of its own."""
    out = []
    i = 0
    n = len(basis)
    while i < n:
        f0 = basis[i]
        comps = _components(f0.l)
        ok = i + len(comps) <= n
        if ok:
            for k, comp in enumerate(comps):
                fk = basis[i + k]
                if (fk.l, fk.x, fk.y, fk.z, tuple(fk.cartesian)) != (f0.l, f0.x, f0.y, f0.z, comp) or \
                        fk.exponents != f0.exponents:
                    ok = False
                    break
                r = np.asarray(fk.coefficients) / np.asarray(f0.coefficients)
                if not np.allclose(r, r[0], rtol=1e-13, atol=0.0):
                    ok = False
                    break
        if ok:
            scales = [basis[i + k].coefficients[0] / f0.coefficients[0] for k in range(len(comps))]
            out.append((_shell_of(f0), [(k, i + k, scales[k]) for k in range(len(comps))]))
            i += len(comps)
        else:
            out.append((_shell_of(f0), [(comps.index(tuple(f0.cartesian)), i, 1.0)]))
            i += 1
    return out


def _pair(A: _Sh, B: _Sh):
    """Primitive-pair quantities with axes (i, j): p, P, K_AB and the per-dimension E tables."""
    a = A.a[:, None]
    b = B.a[None, :]
    p = a + b
    Pc = (a[..., None] * A.c + b[..., None] * B.c) / p[..., None]
    d = A.c - B.c
    K = np.exp(-a * b / p * float(d @ d))
    E = [hermite_e(A.l, B.l, a, b, d[x]) for x in range(3)]
    return p, Pc, K, E


def eri3_block(A: _Sh, B: _Sh, C: _Sh) -> np.ndarray:
    """(ab|c) for every component triple of contracted shells A, B, C: (ncA, ncB, ncC)."""
    p, Pc, K, E = _pair(A, B)
    q = C.a
    p3 = p[:, :, None]
    q3 = q[None, None, :]
    alpha = p3 * q3 / (p3 + q3)
    XPC = Pc[:, :, None, :] - C.c
    L = A.l + B.l + C.l
    R = hermite_r(L, alpha, XPC[..., 0], XPC[..., 1], XPC[..., 2])
    pref = 2.0 * math.pi ** 2.5 / (p3 * q3 * np.sqrt(p3 + q3)) * K[:, :, None]
    w = A.k[:, None, None] * B.k[None, :, None] * C.k[None, None, :] * pref
    # single-centre Hermite expansion of the aux function (b = 0 at its own centre)
    Ec = [hermite_e(C.l, 0, q, 0.0 * q, 0.0) for _ in range(3)]
    ca, cb, cc = _components(A.l), _components(B.l), _components(C.l)
    out = np.zeros((len(ca), len(cb), len(cc)))
    for ic, (lx, ly, lz) in enumerate(cc):
        # G[t,u,v] = sum_{tau,nu,phi} (-1)^(tau+nu+phi) Ec Ec Ec R[t+tau, u+nu, v+phi]
        G = {}
        for t in range(A.l + B.l + 1):
            for u in range(A.l + B.l + 1 - t):
                for v in range(A.l + B.l + 1 - t - u):
                    g = 0.0
                    for tau in range(lx + 1):
                        for nu in range(ly + 1):
                            for phi in range(lz + 1):
                                sgn = -1.0 if (tau + nu + phi) % 2 else 1.0
                                g = g + sgn * Ec[0][lx][0][tau][None, None, :] * Ec[1][ly][0][nu][None, None, :] * \
                                    Ec[2][lz][0][phi][None, None, :] * R[(t + tau, u + nu, v + phi)]
                    G[(t, u, v)] = g
        for ia, (ax, ay, az) in enumerate(ca):
            for ib, (bx, by, bz) in enumerate(cb):
                acc = 0.0
                for t in range(ax + bx + 1):
                    ex = E[0][ax][bx][t][:, :, None]
                    for u in range(ay + by + 1):
                        ey = E[1][ay][by][u][:, :, None]
                        for v in range(az + bz + 1):
                            acc = acc + ex * ey * E[2][az][bz][v][:, :, None] * G[(t, u, v)]
                out[ia, ib, ic] = float((w * acc).sum())
    return out


def _unit_s(center) -> _Sh:
    s = _Sh(center, 0, [0.0], [1.0])
    s.k = np.array([1.0])
    return s


def aux_metric(aux_basis) -> np.ndarray:
    """(P|Q) over the auxiliary functions (src/AO_ints/ThreeCenterIntegrals.cpp:140-161)."""
    blocks = _shell_blocks(aux_basis)
    n = len(aux_basis)
    M = np.zeros((n, n))
    for sa, (A, ma) in enumerate(blocks):
        for (C, mc) in blocks[sa:]:
            blk = eri3_block(A, _unit_s(A.c), C)[:, 0, :]
            for ka, fa, sca in ma:
                for kc, fc, scc in mc:
                    v = blk[ka, kc] * sca * scc
                    M[fa, fc] = v
                    M[fc, fa] = v
    return M


def three_center_raw(basis, aux_basis) -> np.ndarray:
    """raw[P, p n + q] = (pq|P) (src/AO_ints/ThreeCenterIntegrals.cpp:163-184)."""
    ob = _shell_blocks(basis)
    ab = _shell_blocks(aux_basis)
    n, naux = len(basis), len(aux_basis)
    raw = np.zeros((naux, n * n))
    for ia, (A, ma) in enumerate(ob):
        for (B, mb) in ob[ia:]:
            for (C, mc) in ab:
                blk = eri3_block(A, B, C)
                for ka, fa, sa in ma:
                    for kb, fb, sb in mb:
                        for kc, fc, sc in mc:
                            v = blk[ka, kb, kc] * sa * sb * sc
                            raw[fc, fa * n + fb] = v
                            raw[fc, fb * n + fa] = v
    return raw


def _one_e_block(A: _Sh, B: _Sh, kind: str, charges=None) -> np.ndarray:
    p, Pc, K, E = _pair(A, B)
    ca, cb = _components(A.l), _components(B.l)
    w = A.k[:, None] * B.k[None, :] * K
    out = np.zeros((len(ca), len(cb)))
    if kind == "nuclear":
        L = A.l + B.l
        Rs = []
        for (Z, centre) in charges:
            X = Pc - np.asarray(centre)
            Rs.append((Z, hermite_r(L, p, X[..., 0], X[..., 1], X[..., 2])))
    if kind == "kinetic":
        # E tables with two more powers on B for the second derivative
        Ek = [hermite_e(A.l, B.l + 2, A.a[:, None], B.a[None, :], (A.c - B.c)[x]) for x in range(3)]
    sq = np.sqrt(math.pi / p)
    for ia, ax in enumerate(ca):
        for ib, bx in enumerate(cb):
            if kind == "overlap":
                v = E[0][ax[0]][bx[0]][0] * E[1][ax[1]][bx[1]][0] * E[2][ax[2]][bx[2]][0] * sq ** 3
            elif kind == "kinetic":
                b = B.a[None, :]

                def s1(d, i, j):
                    return Ek[d][i][j][0] * sq if j >= 0 else 0.0

                def t1(d, i, j):
                    v = -2.0 * b * b * s1(d, i, j + 2) + b * (2 * j + 1) * s1(d, i, j)
                    if j >= 2:
                        v = v - 0.5 * j * (j - 1) * s1(d, i, j - 2)
                    return v
                sx = [s1(d, ax[d], bx[d]) for d in range(3)]
                tx = [t1(d, ax[d], bx[d]) for d in range(3)]
                v = tx[0] * sx[1] * sx[2] + sx[0] * tx[1] * sx[2] + sx[0] * sx[1] * tx[2]
            else:
                v = 0.0
                for Z, R in Rs:
                    acc = 0.0
                    for t in range(ax[0] + bx[0] + 1):
                        for u in range(ax[1] + bx[1] + 1):
                            for vv in range(ax[2] + bx[2] + 1):
                                acc = acc + E[0][ax[0]][bx[0]][t] * E[1][ax[1]][bx[1]][u] * \
                                    E[2][ax[2]][bx[2]][vv] * R[(t, u, vv)]
                    v = v - Z * 2.0 * math.pi / p * acc
            out[ia, ib] = float((w * v).sum())
    return out


def _one_e(basis, kind, charges=None) -> np.ndarray:
    ob = _shell_blocks(basis)
    n = len(basis)
    M = np.zeros((n, n))
    for ia, (A, ma) in enumerate(ob):
        for (B, mb) in ob[ia:]:
            blk = _one_e_block(A, B, kind, charges)
            for ka, fa, sa in ma:
                for kb, fb, sb in mb:
                    v = blk[ka, kb] * sa * sb
                    M[fa, fb] = v
                    M[fb, fa] = v
    return M


def overlap_matrix(basis) -> np.ndarray:
    """<p|q> (libcint cint1e_ovlp_cart per pair, src/AO_ints/Integrals.cpp:64-129, 189-198)."""
    return _one_e(basis, "overlap")


def kinetic_matrix(basis) -> np.ndarray:
    """<p| -1/2 nabla^2 |q> (src/AO_ints/SchrodingerKinetic.cpp)."""
    return _one_e(basis, "kinetic")


def nuclear_attraction_matrix(basis, charges) -> np.ndarray:
    """<p| -sum_C Z_C / |r - C| |q>; charges = [(Z, (x, y, z))] in bohr (src/AO_ints/NuclearAttraction.cpp)."""
    return _one_e(basis, "nuclear", charges)
