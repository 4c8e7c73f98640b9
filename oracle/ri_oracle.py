"""CPU restatement of the reference's RI hot path in numpy (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this
module, and only as the checker.  The product path (``rerdmft_b200`` + ``librr_ri.so``)
never calls it.

Every function restates one reference function and cites the file:line it follows.  The
restatement is pinned twice: against golden fixtures produced by the reference itself
(``tests/golden/``, made by ``tests/golden/make_golden.py`` from ``oracle/_ref``), and,
where ``oracle/_ref/librrref.so`` is built, against the compiled reference on fresh
random inputs (``tests/test_oracle_vs_reference.py``).

Conventions (reference ``Matrix<T>``, src/Matrix.h:13): row-major; ``B`` is
``(naux, n*n)`` with ``B[P, m*n + k] = (mk|P)``; complex matrices are complex128.
"""
from __future__ import annotations

import numpy as np

# --------------------------------------------------------------------------- linear algebra


def diagonalize(a: np.ndarray):
    """Eigenvalues ascending + eigenvectors in columns (LinearAlgebra.cpp:51 / :122)."""
    return np.linalg.eigh(a)


def canonical_orthogonalize(s: np.ndarray, threshold: float = 1e-10) -> np.ndarray:
    """src/Linear_Algebra/LinearAlgebra.cpp:267-310: keep eigenvalues > threshold,
    X = U_keep w^-1/2, symmetrised back (X U^T) when nothing is dropped."""
    w, u = np.linalg.eigh(s)
    keep = np.nonzero(w > threshold)[0]
    x = u[:, keep] / np.sqrt(w[keep])
    if keep.size == w.size:
        x = x @ u.T
    return x


def canonical_orthogonalize_hermitian(s: np.ndarray, threshold: float = 1e-10) -> np.ndarray:
    """src/Linear_Algebra/LinearAlgebra.cpp:312-349: Jacobi-preconditioned S' = D^-1 S D^-1,
    keep eigenvalues of S' > threshold, X = D^-1 U_keep w^-1/2 (never symmetrised)."""
    d = np.sqrt(np.real(np.diag(s)))
    sp = s / np.outer(d, d)
    w, u = np.linalg.eigh(sp)
    keep = np.nonzero(w > threshold)[0]
    return (u[:, keep] / np.sqrt(w[keep])) / d[:, None]


def three_center_tensor(raw: np.ndarray, metric_x: np.ndarray) -> np.ndarray:
    """src/AO_ints/ThreeCenterIntegrals.cpp:219-236 (riThreeCenterTensor after the libcint integrals):
    B = metric_x^T raw, (naux_kept, n^2)."""
    if raw.shape[0] != metric_x.shape[0]:
        raise ValueError("riThreeCenterTensor: metric_x row count does not match the raw aux basis size")
    return metric_x.T @ raw


def transform_ao_legs(eri3_in: np.ndarray, n_ao: int, t: np.ndarray) -> np.ndarray:
    """src/AO_ints/ThreeCenterIntegrals.cpp:191-217 (transformRiThreeCenterAoLegs): per aux row P,
    u = t^T B^P, out_P = u t."""
    if eri3_in.shape[1] != n_ao * n_ao:
        raise ValueError("transformRiThreeCenterAoLegs: eri3_in column count does not match n_ao^2")
    if t.shape[0] != n_ao:
        raise ValueError("transformRiThreeCenterAoLegs: t row count does not match n_ao")
    naux, n_out = eri3_in.shape[0], t.shape[1]
    b = eri3_in.reshape(naux, n_ao, n_ao)
    return np.einsum("ai,Pab,bj->Pij", t, b, t, optimize=True).reshape(naux, n_out * n_out)


# --------------------------------------------------------------------------- occupied recovery


def _recover_occupied(x: np.ndarray, s: np.ndarray, density: np.ndarray, scale: float):
    """Eigen-decompose X^dagger (S P S * scale) X and keep eigenvalues > 0.5
    (NonRelFockMatrixRi.cpp:96-108 with scale 1/2; X2C_FockMatrixRi.cpp:109-123 and
    UkbFockMatrixRi.cpp:195-209 with scale 1).  Returns (C_occ = X Y_occ, eigenvalues)."""
    sps = (s @ density @ s) * scale
    p_eff = x.conj().T @ sps @ x
    w, y = np.linalg.eigh(p_eff)
    idx = np.nonzero(w > 0.5)[0]
    return x @ y[:, idx], w[idx]


# --------------------------------------------------------------------------- Fock builds


def j_contract(B: np.ndarray, p_flat: np.ndarray) -> np.ndarray:
    """gamma = B vec(P), J = B^T gamma (NonRelFockMatrixRi.cpp:87-92)."""
    return B.T @ (B @ p_flat)


def nonrel_fock(h, B, D, S, X):
    """src/NON_REL/NonRelFockMatrixRi.cpp:71-143: F = h + J - K/2, K from the recovered
    occupied orbitals with c_t = sqrt(2) C_occ^T, tmp_P = c_t B^P, K = sum_P tmp_P^T tmp_P."""
    n = h.shape[0]
    naux = B.shape[0]
    j = j_contract(B, D.reshape(-1)).reshape(n, n)
    c_occ, _ = _recover_occupied(X, S, D, 0.5)
    c_t = np.sqrt(2.0) * c_occ.T  # (nocc, n)
    b3 = B.reshape(naux, n, n)
    tmp = np.einsum("iq,Pqr->Pir", c_t, b3, optimize=True)  # (naux, nocc, n)
    k = np.einsum("Pip,Pir->pr", tmp, tmp, optimize=True)
    return h + j - 0.5 * k


def _k_blocks(slices, c_t_list, pairs):
    """K_fu(a,b) = sum_P sum_i conj(tmp_f(i,a)) tmp_u(i,b), tmp_f = c_t_f B_f^P
    (X2C_FockMatrixRi.cpp:150-181; UkbFockMatrixRi.cpp:118-152)."""
    tmps = [np.einsum("iq,Pqr->Pir", c, b, optimize=True) for c, b in zip(c_t_list, slices)]
    out = {}
    for f, u in pairs:
        out[(f, u)] = np.einsum("Pia,Pib->ab", np.conj(tmps[f]), tmps[u], optimize=True)
    return out


def x2c_fock(h, B, P, S, X):
    """src/X2C_DHF/X2C_FockMatrixRi.cpp:79-205 (two spin blocks [alpha; beta], real B)."""
    n = h.shape[0]
    nl = n // 2
    naux = B.shape[0]
    p_tot = (P[:nl, :nl] + P[nl:, nl:]).real
    j = j_contract(B, p_tot.reshape(-1)).reshape(nl, nl)
    c_occ, occ = _recover_occupied(X, S, P, 1.0)
    sq = np.sqrt(occ)
    c_t = [np.conj(c_occ[off:off + nl, :]).T * sq[:, None] for off in (0, nl)]
    b3 = B.reshape(naux, nl, nl)
    pairs = [(0, 0), (1, 1), (0, 1)]
    kb = _k_blocks([b3, b3], c_t, pairs)
    kb[(1, 0)] = kb[(0, 1)].conj().T
    fock = np.zeros((n, n), dtype=complex)
    fock[:nl, :nl] += j
    fock[nl:, nl:] += j
    for (f, u), k in kb.items():
        fock[f * nl:(f + 1) * nl, u * nl:(u + 1) * nl] -= k
    return h + fock


def ukb_two_electron(nl, ns, B_LL, B_SS, P_ukb, C_occ, occ):
    """src/UKB/UkbFockMatrixRi.cpp:35-183: four flavours [L-alpha, L-beta, S-alpha, S-beta],
    shared gamma from LL and SS, 10 unique K blocks f <= u with K_uf = K_fu^dagger."""
    naux = B_LL.shape[0]
    off = [0, nl, 2 * nl, 2 * nl + ns]
    fs = [nl, nl, ns, ns]
    nu = 2 * nl + 2 * ns
    pL = (P_ukb[0:nl, 0:nl] + P_ukb[nl:2 * nl, nl:2 * nl]).real
    pS = (P_ukb[2 * nl:2 * nl + ns, 2 * nl:2 * nl + ns] + P_ukb[2 * nl + ns:, 2 * nl + ns:]).real
    gamma = B_LL @ pL.reshape(-1) + B_SS @ pS.reshape(-1)
    jL = (B_LL.T @ gamma).reshape(nl, nl)
    jS = (B_SS.T @ gamma).reshape(ns, ns)
    sq = np.sqrt(np.asarray(occ, dtype=float))
    c_t = [np.conj(C_occ[off[f]:off[f] + fs[f], :]).T * sq[:, None] for f in range(4)]
    bl = B_LL.reshape(naux, nl, nl)
    bs = B_SS.reshape(naux, ns, ns)
    pairs = [(0, 0), (1, 1), (2, 2), (3, 3), (0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    kb = _k_blocks([bl, bl, bs, bs], c_t, pairs)
    g = np.zeros((nu, nu), dtype=complex)
    g[0:nl, 0:nl] += jL
    g[nl:2 * nl, nl:2 * nl] += jL
    g[2 * nl:2 * nl + ns, 2 * nl:2 * nl + ns] += jS
    g[2 * nl + ns:, 2 * nl + ns:] += jS
    for (f, u), k in kb.items():
        g[off[f]:off[f] + fs[f], off[u]:off[u] + fs[u]] -= k
        if f != u:
            g[off[u]:off[u] + fs[u], off[f]:off[f] + fs[f]] -= k.conj().T
    return g


def rkb_fock(h, nl, ns, B_LL, B_SS, v_total, s_full, x_full, P):
    """src/UKB/UkbFockMatrixRi.cpp:185-216: occupied recovery in the RKB basis, embed with
    v_total, two-electron part in the UKB basis, project back with v_total^dagger (.) v_total."""
    c_occ_rkb, occ = _recover_occupied(x_full, s_full, P, 1.0)
    c_occ_ukb = v_total @ c_occ_rkb
    p_ukb = v_total @ (P @ v_total.conj().T)
    g = ukb_two_electron(nl, ns, B_LL, B_SS, p_ukb, c_occ_ukb, occ)
    return h + v_total.conj().T @ (g @ v_total)


# --------------------------------------------------------------------------- MO transforms


def nonrel_mo_build(B, C):
    """src/NON_REL/NonRelSpinRiMoEri.cpp:13-43: B_mo^P = C^T B^P C."""
    n = C.shape[0]
    b3 = B.reshape(-1, n, n)
    return np.einsum("ap,Pab,bq->Ppq", C, b3, C, optimize=True).reshape(B.shape[0], -1)


def nonrel_mo_rotated(Bmo, n, U, tolerance=1e-3):
    """src/NON_REL/NonRelSpinRiMoEri.cpp:45-95: U is 2n x 2n, must be blockdiag(u, u) to
    within 1e-3; the two spin blocks are averaged, then B' = u^T B u."""
    off = max(np.abs(U[:n, n:]).max(initial=0.0), np.abs(U[n:, :n]).max(initial=0.0))
    mism = np.abs(U[n:, n:] - U[:n, :n]).max(initial=0.0)
    if off > tolerance or mism > tolerance:
        raise ValueError("rotation is not spin-restricted")
    u = 0.5 * (U[:n, :n] + U[n:, n:])
    return nonrel_mo_build(Bmo, u)


def nonrel_mo_embedded(Bmo, n):
    """src/NON_REL/NonRelSpinRiMoEri.h:77-89: block-diagonal (alpha, beta) embedding."""
    naux = Bmo.shape[0]
    out = np.zeros((naux, 2 * n, 2 * n))
    b3 = Bmo.reshape(naux, n, n)
    out[:, :n, :n] = b3
    out[:, n:, n:] = b3
    return out.reshape(naux, -1)


def nonrel_mo_eri(Bmo, n, abcd):
    """src/NON_REL/NonRelSpinRiMoEri.h:40-50: spin selection, then sum_P B(P,ac) B(P,bd)."""
    out = []
    for a, b, c, d in np.asarray(abcd).reshape(-1, 4):
        if a // n != c // n or b // n != d // n:
            out.append(0.0)
            continue
        ac = (a % n) * n + (c % n)
        bd = (b % n) * n + (d % n)
        out.append(float(Bmo[:, ac] @ Bmo[:, bd]))
    return np.array(out)


def ri_mo_build(nl, ns, B_LL, B_SS, c_ukb):
    """src/UKB/RiMoEri.cpp:64-86 (+ transformBlock :20-60): B(P,p,q) = sum over the four
    UKB blocks of sum_{mu,nu} conj(C(mu,p)) C(nu,q) (mu nu|P)."""
    off = [0, nl, 2 * nl, 2 * nl + ns]
    fs = [nl, nl, ns, ns]
    naux = B_LL.shape[0]
    nt = c_ukb.shape[1]
    out = np.zeros((naux, nt, nt), dtype=complex)
    for f in range(4):
        cb = c_ukb[off[f]:off[f] + fs[f], :]
        b3 = (B_LL if f < 2 else B_SS).reshape(naux, fs[f], fs[f])
        out += np.einsum("ap,Pab,bq->Ppq", np.conj(cb), b3, cb, optimize=True)
    return out.reshape(naux, -1)


def ri_mo_rotated(Bmo, n, U):
    """src/UKB/RiMoEri.cpp:88-110: B' = U^dagger B U per aux index."""
    b3 = Bmo.reshape(-1, n, n)
    return np.einsum("ap,Pab,bq->Ppq", np.conj(U), b3, U, optimize=True).reshape(Bmo.shape[0], -1)


def ri_mo_positive(Bmo, n, off):
    """src/UKB/RiMoEri.cpp:112-120: restrict both MO legs to [off, n)."""
    b3 = Bmo.reshape(-1, n, n)
    return np.ascontiguousarray(b3[:, off:, off:]).reshape(Bmo.shape[0], -1)


def ri_mo_eri(Bmo, n, abcd):
    """src/UKB/RiMoEri.h:50-57: eri(a,b,c,d) = sum_P B(P,a,c) B(P,b,d) (no conjugation)."""
    out = []
    for a, b, c, d in np.asarray(abcd).reshape(-1, 4):
        out.append(Bmo[:, a * n + c] @ Bmo[:, b * n + d])
    return np.array(out)


def jkl_matrices(Bmo, n, pair_of=None):
    """J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i), L_ij = eri(ibar,j,j,ibar) for an MO-RI tensor
    (src/UKB/RiMoEri.h:50 read as in src/Occ_opt/PNOFs.cpp:306-321): J_ij = sum_P B(P,ii) B(P,jj),
    K_ij = sum_P B(P,ij) B(P,ji), L_ij = sum_P B(P,ibar j) B(P,j ibar)."""
    b3 = Bmo.reshape(-1, n, n)
    diag = np.einsum("Pii->Pi", b3)
    J = diag.T @ diag
    K = np.einsum("Pij,Pji->ij", b3, b3, optimize=True)
    L = None
    if pair_of is not None:
        po = np.asarray(pair_of)
        pb = b3[:, po, :]  # [P, i, j] = B(P, ibar, j)
        qb = np.transpose(b3[:, :, po], (0, 2, 1))  # [P, i, j] = B(P, j, ibar)
        L = np.einsum("Pij,Pij->ij", pb, qb, optimize=True)
    return J, K, L


# --------------------------------------------------------------------------- generalized Fock


def hx_fock(h, Bmo, occ, h2, x2, pair_of=None, l1=None, l2=None):
    """src/Hessian_opt/RiGemmFock.cpp:92-157 riHxFockGemm:
    F(p,q) = occ_q h(q,p) + sum_s [h2(s,q) eri(q,s,p,s) - x2(q,s) eri(q,s,s,p)]
             + sum_s 2 eri(s,sbar,qbar,p) (l1(s,qbar) + l2(s,q)),  eri(a,b,c,d)=sum_P B(P,a,c)B(P,b,d)."""
    n = h.shape[0]
    b3 = Bmo.reshape(-1, n, n)
    occ = np.asarray(occ, dtype=float)
    f = (occ[None, :] * h.T).astype(np.result_type(h, Bmo))
    bdiag = np.einsum("Pss->Ps", b3)
    w = bdiag @ h2  # W(P,q) = sum_s Bdiag(P,s) h2(s,q)
    f = f + np.einsum("Pqp,Pq->pq", b3, w, optimize=True)
    # Y(P,t,q) = -x2(q,t) B(P,q,t) [+ 2 (l1(st,qbar) + l2(st,q)) B(P,st,qbar)], F += sum_{P,t} B(P,t,p) Y(P,t,q)
    y = -x2.T[None, :, :] * np.transpose(b3, (0, 2, 1))
    if pair_of is not None:
        po = np.asarray(pair_of)
        st = po  # st = pair_of[t]
        coef = 2.0 * (l1[np.ix_(st, po)] + l2[st, :])  # (t, q): l1(st, qbar) + l2(st, q)
        y = y + coef[None, :, :] * b3[:, st, :][:, :, po]
    f = f + np.einsum("Ptp,Ptq->pq", b3, y, optimize=True)
    return f


# --------------------------------------------------------------------------- DIIS


def commutator_error(F, P, S):
    """src/Utils/DIIS.cpp:53-60: e = F P S - S P F."""
    return F @ (P @ S) - (S @ P) @ F


def _solve_dense(m, rhs, tol):
    """DIIS.cpp:18-48: Gaussian elimination with partial pivoting; None if the pivot ratio
    min|pivot| / max|pivot| is not above `tol`."""
    m = np.array(m, dtype=float)
    rhs = np.array(rhs, dtype=float)
    n = rhs.size
    piv = np.zeros(n)
    for k in range(n):
        best = k + int(np.argmax(np.abs(m[k:, k])))
        if abs(m[best, k]) <= abs(m[k, k]):
            best = k
        if best != k:
            m[[k, best]] = m[[best, k]]
            rhs[[k, best]] = rhs[[best, k]]
        piv[k] = abs(m[k, k])
        if piv[k] == 0.0:
            return None
        for i in range(k + 1, n):
            f = m[i, k] / m[k, k]
            m[i, k:] -= f * m[k, k:]
            rhs[i] -= f * rhs[k]
    if not piv.min() > tol * piv.max():
        return None
    x = np.zeros(n)
    for i in range(n - 1, -1, -1):
        x[i] = (rhs[i] - m[i, i + 1:] @ x[i + 1:]) / m[i, i]
    return x


class Diis:
    """src/Utils/DIIS.cpp:68-131 Diis<T>: newest-first history of at most max_vectors pairs,
    B_ij = Re<e_i|e_j> scaled by its largest diagonal, bordered solve, drop the oldest pair on a
    singular system, input returned unchanged with < 2 pairs."""

    def __init__(self, max_vectors: int):
        self.max_vectors = max_vectors
        self.errors: list = []
        self.values: list = []
        self.last_weights: list = []

    def extrapolate(self, error, value):
        self.last_weights = []
        if self.max_vectors < 2:
            return value
        self.errors.insert(0, np.array(error))
        self.values.insert(0, np.array(value))
        del self.errors[self.max_vectors:]
        del self.values[self.max_vectors:]
        total = len(self.errors)
        bf = np.empty((total, total))
        for i in range(total):
            for j in range(i, total):
                bf[i, j] = bf[j, i] = float(np.real(np.vdot(self.errors[i], self.errors[j])))
        for m in range(total, 1, -1):
            scale = max(bf[i, i] for i in range(m))
            if not scale > 0.0:
                return value
            a = np.zeros((m + 1, m + 1))
            a[:m, :m] = bf[:m, :m] / scale
            a[:m, m] = a[m, :m] = -1.0
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            x = _solve_dense(a, rhs, 1e-14)
            if x is None:
                continue
            res = np.zeros_like(self.values[0])
            for i in range(m):
                res = res + x[i] * self.values[i]
            self.last_weights = list(x[:m])
            return res
        return value


# --------------------------------------------------------------------------- SCF loops


def _kramers_even(m, blocks):
    n = m.shape[0]
    nb = n // blocks
    idx = np.arange(n)
    blk = idx // nb
    partner = (blk ^ 1) * nb + idx % nb
    sign = np.where(blk % 2 == 0, 1.0, -1.0)
    return 0.5 * (m + np.outer(sign, sign) * np.conj(m[np.ix_(partner, partner)]))


def _scf(fock_fn, h, x, s, p0, density_fn, diis_size, max_iter, e_tol, d_tol, restrict=None):
    """Shared body of NonRelHartreeFock.cpp:117-198, X2C_HF.cpp:43-138, C4_DHF.cpp:45-142:
    F(P) -> DIIS(e = FPS - SPF) -> X^dagger F X -> eig -> C = X U -> P_new;
    E = 1/2 Tr[P_cur (h + F)] with the un-extrapolated F; converged when dP < d_tol OR
    dE < e_tol (from the second iteration); DIIS replaces mixing (p_current = p_new)."""
    restrict = restrict or (lambda p: p)
    p_cur = restrict(p0)
    prev = 0.0
    use_diis = diis_size >= 2
    diis = Diis(diis_size if use_diis else 0)
    hist = []
    converged = False
    it = 0
    for it in range(1, max_iter + 1):
        f = fock_fn(p_cur)
        f_scf = diis.extrapolate(commutator_error(f, p_cur, s), f) if use_diis else f
        w, u = np.linalg.eigh(x.conj().T @ f_scf @ x)
        c = x @ u
        p_new = restrict(density_fn(c))
        e = 0.5 * float(np.real(np.trace(p_cur @ (h + f))))
        dp = float(np.abs(p_new - p_cur).max())
        de = abs(e - prev)
        hist.append(e)
        if it > 1 and (dp < d_tol or de < e_tol):
            converged = True
            prev = e
            break
        prev = e
        p_cur = p_new
    return dict(energy=hist[-1], iterations=it, converged=converged, P=p_cur, history=np.array(hist))


def nonrel_scf(sysd, diis_size=5, max_iter=100, e_tol=1e-8, d_tol=1e-6):
    """src/NON_REL/NonRelHartreeFock.cpp:117-198 (RI overload :219); density = 2 C_occ C_occ^T
    over the lowest n_electrons/2 columns (:42-69)."""
    h, B, S, X = sysd["h"], sysd["B"], sysd["S"], sysd["X"]
    nocc = sysd["n_electrons"] // 2

    def dens(c):
        return 2.0 * c[:, :nocc] @ c[:, :nocc].T

    return _scf(lambda p: nonrel_fock(h, B, p, S, X), h, X, S, sysd["D0"], dens, diis_size, max_iter, e_tol, d_tol)


def x2c_scf(sysd, diis_size=5, max_iter=100, e_tol=1e-8, d_tol=1e-6, kramers=True):
    """src/X2C_DHF/X2C_HF.cpp:43-138 with x2cDensityMatrix (X2C_DensityMatrix.cpp:8) and the
    kramersSymmetrizeAo projection (KramersPairing.cpp:320) when n_electrons is even."""
    h, B, S, X = sysd["h"], sysd["B"], sysd["S"], sysd["X"]
    ne = sysd["n_electrons"]
    restrict = (lambda p: _kramers_even(p, 2)) if (kramers and ne % 2 == 0) else None

    def dens(c):
        return c[:, :ne] @ c[:, :ne].conj().T

    return _scf(lambda p: x2c_fock(h, B, p, S, X), h, X, S, sysd["P0"], dens, diis_size, max_iter, e_tol, d_tol,
                restrict)


def dhf_scf(sysd, diis_size=5, max_iter=100, e_tol=1e-8, d_tol=1e-6, kramers=True):
    """src/C4_DHF/C4_DHF.cpp:45-142 with rkbDensityMatrix (RkbDensityMatrix.cpp:16: occupied
    spinors start at n/2) and kramersSymmetrizeRkbAo (KramersPairing.cpp:351)."""
    h = sysd["h"]
    args = (sysd["nl"], sysd["ns"], sysd["B_LL"], sysd["B_SS"], sysd["v_total"], sysd["s_full"], sysd["x_full"])
    ne = sysd["n_electrons"]
    restrict = (lambda p: _kramers_even(p, 4)) if (kramers and ne % 2 == 0) else None

    def dens(c):
        n0 = c.shape[0] // 2
        cc = c[:, n0:n0 + ne]
        return cc @ cc.conj().T

    return _scf(lambda p: rkb_fock(h, *args, p), h, sysd["x_full"], sysd["s_full"], sysd["P0"], dens, diis_size,
                max_iter, e_tol, d_tol, restrict)


# --------------------------------------------------------------------------- orbital rotations


def adam_step_sequence(grads, lr=0.01, b1=0.7, b2=0.9, eps=1e-15):
    """Adam<T>::step (src/Utils/ADAM.cpp:33-51): AMSGrad-style moments; complex entries share one
    real second moment |g|^2 (the step keeps the direction of the complex gradient)."""
    grads = np.asarray(grads)
    m1 = np.zeros(grads.shape[1], dtype=grads.dtype)
    m2 = np.zeros(grads.shape[1])
    mx = np.zeros(grads.shape[1])
    out = np.empty_like(grads)
    for t, g in enumerate(grads, start=1):
        c1, c2 = 1.0 - b1 ** t, 1.0 - b2 ** t
        m1 = b1 * m1 + (1.0 - b1) * g
        m2 = b2 * m2 + (1.0 - b2) * np.abs(g) ** 2
        mx = np.maximum(mx, m2 / c2)
        out[t - 1] = -lr * (m1 / c1) / (np.sqrt(mx) + eps)
    return out


def pair_indices(n):
    """adamPairIndices(n) (src/Utils/ADAM.cpp:57): (1,0), (2,0), (2,1), (3,0), ..."""
    return [(p, q) for p in range(n) for q in range(p)]


def kappa_matrix(n, pairs, step):
    """adamKappaMatrix (ADAM.cpp:92-128): kappa_pq = step, kappa_qp = -conj(step)."""
    k = np.zeros((n, n), dtype=np.result_type(step, float))
    for (p, q), s in zip(pairs, step):
        k[p, q] = s
        k[q, p] = -np.conj(s)
    return k


def rotation_matrix(kappa):
    """exp(-kappa) for anti-Hermitian kappa via the Hermitian i*kappa = V w V^dagger
    (src/Hessian_opt/SpinorRotation.cpp:17-90)."""
    w, v = np.linalg.eigh(1j * kappa)
    u = (v * np.exp(1j * w)) @ v.conj().T
    return u.real if np.isrealobj(kappa) else u


def orbital_gradient(F):
    """g_pq = 2 (F_qp - conj F_pq), lower triangle p >= q (src/Hessian_opt/OrbitalGradient.h)."""
    return np.tril(2.0 * (F.T - np.conj(F)))


def hx_energy_from_fock(h, occ, F):
    """E = 1/2 sum_q [n_q Re h_qq + Re F_qq]: the double-counting identity the reference's rotation
    problem uses with the generalized Fock of hx_fock (src/Full_opt/FullOptimization.cpp:1383)."""
    return 0.5 * float(np.sum(np.asarray(occ) * np.real(np.diag(h))) + np.real(np.trace(F)))


def _eri(b3, a, b, c, d):
    return float(b3[:, a, c] @ b3[:, b, d])


def hx_hessian_diag(h, Bmo, occ, h2, x2, F, pairs, pair_of=None, l1=None, l2=None):
    """hartreeExchangeHessianElement(p,q,p,q) (src/Hessian_opt/HartreeExchangeHessian.cpp:221) for
    real orbitals: the antisymmetrised combination of the bare G_pq,rs terms (:57-118 H/X part,
    :124-161 L1/L2 part) with eri(a,b,c,d) = sum_P B(P,a,c) B(P,b,d).  Pure Python loops: small n."""
    n = h.shape[0]
    b3 = Bmo.reshape(-1, n, n)
    occ = np.asarray(occ, dtype=float)

    def raw(p, q, r, s):
        t = 0.0
        if q == r:
            t += F[p, s]
            t -= h[s, p] * occ[r]
            t += sum(h2[r, u] * (_eri(b3, u, s, p, u) - _eri(b3, s, u, p, u)) for u in range(n))
        if s == p:
            t += F[q, r]
            t -= h[q, r] * occ[p]
            t += sum(h2[p, u] * (_eri(b3, u, q, r, u) - _eri(b3, u, q, u, r)) for u in range(n))
        i1, i2 = _eri(b3, s, q, p, r), _eri(b3, s, q, r, p)
        t += i1 * (x2[r, q] - h2[s, q] + x2[p, s] - x2[r, p])
        t += i2 * (h2[r, p] + x2[q, s] - x2[p, s] - x2[r, q])
        return t

    def raw_l(p, q, r, s):
        po = pair_of
        t = 0.0
        if q == po[s]:
            t -= 2.0 * sum(_eri(b3, u, po[u], p, r) * (l1[u, s] + l2[u, q]) for u in range(n))
        c = l1[r, q] + l2[r, po[q]]
        t += 2.0 * c * (_eri(b3, po[r], s, p, po[q]) - _eri(b3, s, po[r], p, po[q]))
        c = l1[p, s] + l2[p, po[s]]
        t += 2.0 * c * (_eri(b3, po[p], q, r, po[s]) - _eri(b3, po[p], q, po[s], r))
        if p == po[r]:
            t += 2.0 * sum(_eri(b3, s, q, w, po[w]) * (l1[r, w] + l2[r, po[w]]) for w in range(n))
        return t

    out = []
    for p, q in pairs:
        v = raw(p, q, p, q) - raw(p, q, q, p) - raw(q, p, p, q) + raw(q, p, q, p)
        if pair_of is not None:
            v += raw_l(p, q, p, q) - raw_l(p, q, q, p) - raw_l(q, p, p, q) + raw_l(q, p, q, p)
        out.append(v)
    return np.array(out)


class RotationProblemNumpy:
    """RotationProblem (src/Full_opt/FullOptimization.cpp:1330-1548) for RiNonRelSpinMoEri and a
    fixed-occupation hartree-exchange functional: spin-orbital pairs p > q, twin-averaged gradient,
    rotations exp(-kappa) of the spatial block, energy from the generalized-Fock identity."""

    def __init__(self, Bmo, h, occ, h2, x2, pair_of=None, l1=None, l2=None):
        self.n = h.shape[0]
        self.d = 2 * self.n
        self.B, self.h = Bmo.copy(), h.copy()
        self.occ, self.h2, self.x2 = occ, h2, x2
        self.po, self.l1, self.l2 = pair_of, l1, l2
        self.pairs = pair_indices(self.d)
        idx = {pq: i for i, pq in enumerate(self.pairs)}
        self.twin = []
        for p, q in self.pairs:
            pp, qq = (p + self.n) % self.d, (q + self.n) % self.d
            self.twin.append(idx[(pp, qq)] if pp > qq else -1)
        self.best = None

    def spin_h(self):
        H = np.zeros((self.d, self.d))
        H[: self.n, : self.n] = self.h
        H[self.n:, self.n:] = self.h
        return H

    def fock(self):
        return hx_fock(self.spin_h(), nonrel_mo_embedded(self.B, self.n), self.occ, self.h2, self.x2, self.po, self.l1,
                       self.l2)

    def energy(self):
        return hx_energy_from_fock(self.spin_h(), self.occ, self.fock())

    def gradient(self):
        g = orbital_gradient(self.fock())
        raw = np.array([g[p, q] for p, q in self.pairs])
        out = raw.copy()
        for i, t in enumerate(self.twin):
            if t >= 0:
                out[i] = 0.5 * (raw[i] + raw[t])
        return out

    def rotate(self, step):
        k = kappa_matrix(self.d, self.pairs, step)
        u = rotation_matrix(k)[: self.n, : self.n]
        b3 = self.B.reshape(-1, self.n, self.n)
        self.B = np.einsum("ai,Pab,bj->Pij", u, b3, u, optimize=True).reshape(b3.shape[0], -1)
        self.h = u.T @ self.h @ u

    def save_best(self):
        self.best = (self.B.copy(), self.h.copy())

    def restore_best(self):
        self.B, self.h = self.best[0].copy(), self.best[1].copy()


class RotationProblemComplexNumpy:
    """RotationProblem<std::complex<double>, RiMoEri> (src/Full_opt/FullOptimization.cpp:1330-1548) for a
    fixed-occupation hartree-exchange functional: pairs excludeNegative(adamPairIndices(n), n_negative)
    (FullOptimization.cpp:83-92), complex gradient 2 (F_qp - conj F_pq), kappa_pq = step,
    kappa_qp = -conj(step) (ADAM.cpp:106-128), rotations U = exp(-kappa) through the eigenvectors of
    i kappa (SpinorRotation.cpp:17-90) applied as U^dagger B^P U and U^dagger h U, energy from the
    generalized-Fock identity."""

    def __init__(self, Bmo, h, occ, h2, x2, pair_of=None, l1=None, l2=None, n_negative=0):
        self.n = h.shape[0]
        self.B, self.h = np.array(Bmo, dtype=complex), np.array(h, dtype=complex)
        self.occ, self.h2, self.x2 = occ, h2, x2
        self.po, self.l1, self.l2 = pair_of, l1, l2
        self.pairs = [(p, q) for p, q in pair_indices(self.n) if p >= n_negative and q >= n_negative]
        self.u = np.eye(self.n, dtype=complex)
        self.best = None

    def fock(self):
        return hx_fock(self.h, self.B, self.occ, self.h2, self.x2, self.po, self.l1, self.l2)

    def energy(self):
        return hx_energy_from_fock(self.h, self.occ, self.fock())

    def gradient(self):
        F = self.fock()
        return np.array([2.0 * (F[q, p] - np.conj(F[p, q])) for p, q in self.pairs], dtype=complex)

    def rotate(self, step):
        u = rotation_matrix(kappa_matrix(self.n, self.pairs, np.asarray(step, dtype=complex)))
        b3 = self.B.reshape(-1, self.n, self.n)
        self.B = np.einsum("ai,Pab,bj->Pij", u.conj(), b3, u, optimize=True).reshape(b3.shape[0], -1)
        self.h = u.conj().T @ self.h @ u
        self.u = self.u @ u

    def save_best(self):
        self.best = (self.B.copy(), self.h.copy(), self.u.copy())

    def restore_best(self):
        self.B, self.h, self.u = (x.copy() for x in self.best)


class AdamOptimizerNumpy:
    """AdamOptimizer<T>::run (src/Utils/ADAM.cpp:140-213) with the AdamOptions defaults; complex
    gradients take a complex first moment and the second moment of |g|^2 (Adam<complex>::step,
    ADAM.cpp:33-51)."""

    def __init__(self, lr=0.01, rate_factor=0.2, base=10, inc=20, limit=200, gtol=1e-5, etol=1e-9):
        self.opt = dict(lr=lr, rate_factor=rate_factor, base=base, inc=inc, limit=limit, gtol=gtol, etol=etol)
        self.lr, self.extra, self.restart = lr, 0, False

    def run(self, prob):
        o = self.opt
        self.restart = False
        max_calls = o["base"] + self.extra
        if max_calls > o["limit"]:
            max_calls = o["base"]
        n = len(prob.pairs) if hasattr(prob, "pairs") else prob.dim
        m1, m2, mx, t = None, np.zeros(n), np.zeros(n), 0
        e_old = prob.energy()
        e_best = e_old
        prob.save_best()
        improved, ediff = False, 0.0
        while True:
            g = prob.gradient()
            if m1 is None:
                m1 = np.zeros(n, dtype=g.dtype)
            if np.abs(g).max() < o["gtol"]:
                self.lr, self.extra = o["lr"], 0
                break
            t += 1
            c1, c2 = 1 - 0.7 ** t, 1 - 0.9 ** t
            m1 = 0.7 * m1 + 0.3 * g
            sq = g.real * g.real + g.imag * g.imag if np.iscomplexobj(g) else g * g
            m2 = 0.9 * m2 + 0.1 * sq
            mx = np.maximum(mx, m2 / c2)
            prob.rotate(-self.lr * (m1 / c1) / (np.sqrt(mx) + 1e-15))
            e = prob.energy()
            if e < e_best:
                improved, e_best = True, e
                prob.save_best()
            ediff = e - e_old
            if t > 1 and abs(ediff) < o["etol"]:
                break
            e_old = e
            if t == max_calls:
                break
        if not improved and abs(ediff) > o["etol"]:
            self.restart = True
            self.lr *= o["rate_factor"]
            self.extra += o["inc"]
        prob.restore_best()
        return dict(iterations=t, energy_best=e_best, restart_requested=self.restart)


# --------------------------------------------------------------------------- RI sigma-vector primitives


def sigma_toolkit(B: np.ndarray, n: int, K: np.ndarray) -> dict:
    """src/Hessian_opt/RiSigmaHessianToolkit.cpp:24-55: KB1[P] = K B^P, KB2[P] = B^P K (K real, applied
    unconjugated) and the diagonals of B, KB1, KB2."""
    naux = B.shape[0]
    b = B.reshape(naux, n, n)
    kb1 = np.einsum("as,Psb->Pab", K, b, optimize=True)
    kb2 = np.einsum("Par,rb->Pab", b, K, optimize=True)
    d = np.arange(n)
    return dict(kb1=kb1.reshape(naux, n * n), kb2=kb2.reshape(naux, n * n), bdiag=b[:, d, d], kb1diag=kb1[:, d, d],
                kb2diag=kb2[:, d, d])


def _sigma_values(op: dict, n: int, naux: int, dtype) -> np.ndarray:
    """value(P,t,x) of a PairOp (src/Hessian_opt/RiSigmaGemm.h:21-26, fillOp RiSigmaGemm.cpp:38-61):
    s(P, idx(t,x)) * w(t,x) * row(P,t), then right-multiplied by post when given."""
    v = np.ones((naux, n, n), dtype=dtype)
    if op.get("s") is not None:
        v = v * op["s"][:, np.asarray(op["idx"], dtype=np.int64)].reshape(naux, n, n)
    if op.get("w") is not None:
        v = v * np.asarray(op["w"]).reshape(n, n)[None]
    if op.get("row") is not None:
        v = v * op["row"][:, :, None]
    if op.get("post") is not None:
        v = v @ op["post"]
    return v


def sigma_pair_contract(target, sign, n, naux, f, g):
    """pairContract (RiSigmaGemm.cpp:65-95): target(x,y) + sign sum_{P,t} F(P,t,x) G(P,t,y), no
    conjugation (the reference's GEMM is A^T B)."""
    cplx = any(np.iscomplexobj(a) for a in (target, f.get("s"), g.get("s"), f.get("row"), g.get("row"))
               if a is not None)
    dt = np.complex128 if cplx else np.float64
    F = _sigma_values(f, n, naux, dt)
    G = _sigma_values(g, n, naux, dt)
    return target + sign * np.einsum("Ptx,Pty->xy", F, G, optimize=True)


def sigma_diag_contract(target, n, naux, S, Ua=None, Ub=None):
    """diagContract (RiSigmaGemm.cpp:97-114): target(a,b) + sum_P S(P, b n + a) (Ua(P,a) + Ub(P,b))."""
    s = S.reshape(naux, n, n)  # s[P, b, a]
    u = np.zeros((naux, n, n), dtype=np.result_type(S, target))  # [P, b, a]
    if Ua is not None:
        u = u + Ua[:, None, :]
    if Ub is not None:
        u = u + Ub[:, :, None]
    return target + np.einsum("Pba,Pba->ab", s, u, optimize=True)


def sigma_accum_u(U, alpha, n, naux, D, Wm):
    """accumU (RiSigmaGemm.cpp:116-126): U(P,x) + alpha sum_t D[P n + t] Wm(x,t)."""
    return U + alpha * (np.asarray(D).reshape(naux, n) @ Wm.T)


# --------------------------------------------------------------------------- CASSCF RI operators


def _cas_operand(Bmo, n):
    """The tensor the CASSCF RI operators act on (src/MCSCF/CasFock.cpp:246-262): embeddedB for a real
    spatial tensor (NonRelSpinRiMoEri.h:77-89), the tensor itself for a complex one; returns (B, d)."""
    if np.iscomplexobj(Bmo):
        return Bmo, n
    naux = Bmo.shape[0]
    b = Bmo.reshape(naux, n, n)
    e = np.zeros((naux, 2 * n, 2 * n))
    e[:, :n, :n] = b
    e[:, n:, n:] = b
    return e.reshape(naux, 4 * n * n), 2 * n


def cas_two_electron(Bmo, n, rho):
    """riTwoElectronOperator (CasFock.cpp:74-113): G = J - K, c_P = sum_st rho_st B(P,st), J = B^T c,
    K = sum_P B_P conj(rho~) B_P with rho~ = rho's eigen-decomposition without |w| <= 1e-14."""
    B, d = _cas_operand(Bmo, n)
    naux = B.shape[0]
    c = B @ rho.reshape(-1)
    J = (B.T @ c).reshape(d, d)
    w, u = np.linalg.eigh(rho)
    k = np.abs(w) > 1e-14
    rt = (np.conj(u[:, k]) * w[k]) @ u[:, k].T  # conj(U) diag(w) U^T
    b = B.reshape(naux, d, d)
    K = np.einsum("Prt,ts,Psp->rp", b, rt, b, optimize=True)
    return J - K


def cas_cumulant_fock(Bmo, n, active, lam):
    """riActiveCumulantFock (CasFock.cpp:116-133)."""
    B, d = _cas_operand(Bmo, n)
    naux, a = B.shape[0], len(active)
    b = B.reshape(naux, d, d)
    act = np.asarray(active)
    bact = b[:, act][:, :, act].reshape(naux, a * a)
    T = (bact @ np.asarray(lam).reshape(a * a, a * a)).reshape(naux, a, a)  # [P, r, q]
    return np.einsum("Prp,Prq->pq", b[:, act, :], T, optimize=True)


def cas_active_integrals(Bmo, n, active):
    """riActiveIntegrals (CasFock.cpp:136-147): (tu|vw) = sum_P B(P,tu) B(P,vw), flat [t,u,v,w]."""
    B, d = _cas_operand(Bmo, n)
    naux, a = B.shape[0], len(active)
    act = np.asarray(active)
    ba = B.reshape(naux, d, d)[:, act][:, :, act].reshape(naux, a * a)
    return (ba.T @ ba).reshape(-1)
