"""Seeded synthetic inputs for the RI hot path (numpy, host side).

The reference builds its metric-contracted 3-center tensor ``B`` with libcint
(src/AO_ints/ThreeCenterIntegrals.cpp:219 riThreeCenterTensor).  Integral generation is
not part of this library, so benchmarks and tests feed tensors of the same shape and
structure, drawn from a seed:

* AO and auxiliary centres uniform in an ``L``-bohr cube;
* ``B[P, m, n] = c[P, m, n] * exp(-a (|r_m - r_P|^2 + |r_n - r_P|^2))`` with ``c``
  symmetric in (m, n) and N(0, 1) entries (row-major ``(naux, n*n)``, the reference's
  ``eri3_L`` layout, src/NON_REL/NonRelFockMatrixRi.h:32);
* ``D = 2 C_occ C_occ^T`` with ``C_occ`` a QR-orthonormalised Gaussian ``n x nocc``.

``*_system`` helpers add what an SCF loop needs (``h``, ``S``, ``X``, a start density),
chosen so that the closed-shell / Kramers-restricted SCF converges: a core Hamiltonian
with a clear gap after the occupied block and an overlap close to identity.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "ri_tensor", "occupied_density", "canonical_orthogonalize", "nonrel_system",
    "x2c_system", "rkb_system", "kramers_pair_ao", "kramers_even", "random_unitary", "random_orthogonal",
]


def ri_tensor(n: int, naux: int, seed: int, box: float = 20.0, alpha: float = 0.3,
              scale: float = 1.0, rng: np.random.Generator | None = None) -> np.ndarray:
    """(naux, n*n) float64 tensor following the cube/Gaussian recipe above."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    r_ao = rng.uniform(0.0, box, size=(n, 3))
    r_aux = rng.uniform(0.0, box, size=(naux, 3))
    d2 = ((r_aux[:, None, :] - r_ao[None, :, :]) ** 2).sum(-1)  # (naux, n)
    g = np.exp(-alpha * d2)
    out = np.empty((naux, n, n))
    for p in range(naux):
        c = rng.standard_normal((n, n))
        c = (c + c.T) * (0.5 ** 0.5)
        out[p] = c * g[p][:, None] * g[p][None, :]
    out *= scale
    return out.reshape(naux, n * n)


def occupied_density(n: int, nocc: int, rng: np.random.Generator, factor: float = 2.0):
    """(C_occ, D = factor * C_occ C_occ^T) with orthonormal Gaussian C_occ."""
    c, _ = np.linalg.qr(rng.standard_normal((n, nocc)))
    return c, factor * (c @ c.T)


def canonical_orthogonalize(s: np.ndarray, threshold: float = 1e-10) -> np.ndarray:
    """Loewdin canonical orthogonalisation, symmetrised when nothing is dropped
    (same rule as src/Linear_Algebra/LinearAlgebra.cpp:267-310)."""
    w, u = np.linalg.eigh(s)
    keep = w > threshold
    x = u[:, keep] / np.sqrt(w[keep])
    if keep.all():
        x = x @ u.conj().T
    return x


def random_orthogonal(n: int, rng: np.random.Generator) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diag(r))


def random_unitary(n: int, rng: np.random.Generator) -> np.ndarray:
    z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def _core_hamiltonian(n: int, nocc: int, rng: np.random.Generator, gap: float) -> np.ndarray:
    occ = -2.0 + 0.8 * rng.random(nocc)
    vir = gap - 1.2 + 2.5 * rng.random(n - nocc)
    q = random_orthogonal(n, rng)
    return (q * np.concatenate([occ, vir])) @ q.T


def _overlap(n: int, rng: np.random.Generator, eps: float) -> np.ndarray:
    a = rng.standard_normal((n, n))
    return np.eye(n) + eps * (a + a.T) / np.sqrt(n)


def nonrel_system(n: int, naux: int, nocc: int, seed: int, b_scale: float | None = None,
                  box: float = 8.0, overlap_eps: float = 0.05, gap: float = 1.5) -> dict:
    """Closed-shell RHF inputs: B (naux, n^2), h, S, X (canonical), D0 (core guess)."""
    rng = np.random.default_rng(seed)
    B = ri_tensor(n, naux, seed, box=box, rng=rng)
    if b_scale is None:  # two-electron terms of order 0.3 relative to h
        b_scale = 2.4 / max(1e-30, np.sqrt(np.abs(B).max() * np.sqrt(naux)))
    B *= b_scale
    h = _core_hamiltonian(n, nocc, rng, gap)
    S = _overlap(n, rng, overlap_eps)
    X = canonical_orthogonalize(S)
    w, y = np.linalg.eigh(X.T @ h @ X)
    C = X @ y
    D0 = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    return dict(n=n, naux=naux, nocc=nocc, B=B, h=h, S=S, X=X, D0=D0, n_electrons=2 * nocc)


def _kramers_partner(n: int, blocks: int):
    """Partner index and sign of each basis function for time reversal in a layout made of
    `blocks` equal spin blocks alternating alpha/beta (2: [alpha; beta] X2C AO layout,
    src/Utils/KramersPairing.cpp:320; 4: [L-alpha; L-beta; S-alpha; S-beta] RKB layout, :308)."""
    nb = n // blocks
    idx = np.arange(n)
    blk = idx // nb
    partner = (blk ^ 1) * nb + idx % nb
    sign = np.where(blk % 2 == 0, 1.0, -1.0)
    return partner, sign


def kramers_even(m: np.ndarray, blocks: int = 2) -> np.ndarray:
    """Time-reversal-even part (M + Theta M Theta^-1) / 2 in the given block layout."""
    partner, sign = _kramers_partner(m.shape[0], blocks)
    return 0.5 * (m + np.outer(sign, sign) * np.conj(m[np.ix_(partner, partner)]))


def kramers_pair_ao(m: np.ndarray) -> np.ndarray:
    """[alpha AO; beta AO] layout projection (src/Utils/KramersPairing.cpp:320 kramersSymmetrizeAo)."""
    return kramers_even(m, 2)


def _kramers_spectrum(n: int, blocks: int, pair_energies: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """Kramers-even Hermitian matrix whose doubly degenerate spectrum is `pair_energies`."""
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    k = kramers_even(0.5 * (a + a.conj().T), blocks)
    _, v = np.linalg.eigh(k)
    e = np.repeat(np.asarray(pair_energies), 2)
    return (v * e) @ v.conj().T


def x2c_system(nl: int, naux: int, n_electrons: int, seed: int, b_scale: float | None = None,
               box: float = 8.0, gap: float = 1.5) -> dict:
    """X2C-HF inputs in the [alpha; beta] spin-orbital AO basis (dimension 2 nl): real
    B (naux, nl^2), complex Kramers-even h_x2c, S = blockdiag(S_L, S_L), X (symmetric
    canonical), Kramers-even start density P0 (lowest n_electrons spinors of h)."""
    rng = np.random.default_rng(seed)
    B = ri_tensor(nl, naux, seed, box=box, rng=rng)
    if b_scale is None:
        b_scale = 2.4 / max(1e-30, np.sqrt(np.abs(B).max() * np.sqrt(naux)))
    B *= b_scale
    n = 2 * nl
    S_L = _overlap(nl, rng, 0.05)
    S = np.zeros((n, n), dtype=complex)
    S[:nl, :nl] = S_L
    S[nl:, nl:] = S_L
    X = canonical_orthogonalize(S)
    npair_occ = n_electrons // 2
    e = np.concatenate([-2.0 + 0.8 * rng.random(npair_occ), gap - 1.2 + 2.5 * rng.random(nl - npair_occ)])
    h_o = _kramers_spectrum(n, 2, e, rng)
    sx = S @ X
    h = sx @ h_o @ sx.conj().T
    h = kramers_even(0.5 * (h + h.conj().T), 2)
    w, y = np.linalg.eigh(X.conj().T @ h @ X)
    C = X @ y
    P0 = kramers_even(C[:, :n_electrons] @ C[:, :n_electrons].conj().T, 2)
    return dict(nl=nl, naux=naux, B=B, h=h, S=S, X=X, P0=P0, n_electrons=n_electrons)


def rkb_system(nl: int, ns: int, naux: int, n_electrons: int, seed: int, b_scale: float | None = None,
               box: float = 8.0, small_scale: float = 0.05, gap: float = 1.5) -> dict:
    """4-component RKB inputs.  RKB basis [L-alpha, L-beta, S-alpha, S-beta] of dimension
    n_rkb = 4 nl; UKB basis of dimension n_ukb = 2 nl + 2 ns; v_total (n_ukb x n_rkb) embeds
    the large block as the identity and each RKB small function as a combination of UKB small
    functions.  h_rkb has a Dirac-like spectrum: nl*2 negative-energy states far below and the
    positive-energy block with a gap after the occupied spinors."""
    rng = np.random.default_rng(seed)
    B_LL = ri_tensor(nl, naux, seed, box=box, rng=rng)
    B_SS = ri_tensor(ns, naux, seed + 1, box=box, rng=rng)
    if b_scale is None:
        b_scale = 2.4 / max(1e-30, np.sqrt(np.abs(B_LL).max() * np.sqrt(naux)))
    B_LL *= b_scale
    B_SS *= b_scale * small_scale
    n_rkb, n_ukb = 4 * nl, 2 * nl + 2 * ns
    v = np.zeros((n_ukb, n_rkb), dtype=complex)
    v[: 2 * nl, : 2 * nl] = np.eye(2 * nl)
    w_s = (rng.standard_normal((ns, nl)) + 1j * rng.standard_normal((ns, nl))) / np.sqrt(ns)
    v[2 * nl: 2 * nl + ns, 2 * nl: 3 * nl] = w_s
    v[2 * nl + ns:, 3 * nl:] = np.conj(w_s)
    S_ukb = np.eye(n_ukb, dtype=complex)
    S_L = _overlap(nl, rng, 0.05)
    S_ukb[:nl, :nl] = S_L
    S_ukb[nl: 2 * nl, nl: 2 * nl] = S_L
    s_full = v.conj().T @ S_ukb @ v
    s_full = 0.5 * (s_full + s_full.conj().T)
    x_full = canonical_orthogonalize(s_full)
    # Dirac-like one-body operator in the orthonormal basis (Kramers pairs: nl*... negative-energy
    # pairs far below, then the occupied positive-energy pairs, then virtuals), back to the AO basis.
    n_eff = x_full.shape[1]
    npair = n_eff // 2
    npair_neg = npair // 2
    npair_occ = n_electrons // 2
    e = np.concatenate([-60.0 - 5.0 * rng.random(npair_neg), -2.0 + 0.8 * rng.random(npair_occ),
                        gap - 1.2 + 2.5 * rng.random(npair - npair_neg - npair_occ)])
    h_ortho = _kramers_spectrum(n_eff, 4, e, rng)
    sx = s_full @ x_full
    h_rkb = sx @ h_ortho @ sx.conj().T
    h_rkb = kramers_even(0.5 * (h_rkb + h_rkb.conj().T), 4)
    w, y = np.linalg.eigh(x_full.conj().T @ h_rkb @ x_full)
    c = x_full @ y
    occ_cols = c[:, n_eff // 2: n_eff // 2 + n_electrons]
    P0 = kramers_even(occ_cols @ occ_cols.conj().T, 4)
    return dict(nl=nl, ns=ns, naux=naux, B_LL=B_LL, B_SS=B_SS, v_total=v, s_full=s_full, x_full=x_full,
                h=h_rkb, P0=P0, n_electrons=n_electrons, n_rkb=n_rkb, n_ukb=n_ukb)


def functional_system(ns: int, naux: int, seed: int, nocc: int | None = None, with_pairs: bool = False,
                      box: float = 8.0) -> dict:
    """Fixed-occupation functional-stage inputs for the nonrelativistic spin-orbital RI tensor: an
    MO-basis tensor (naux, ns^2) of the cube/Gaussian recipe in a random orthonormal basis, a
    one-electron matrix h with nocc low levels (not diagonal in that basis), natural occupations
    (nocc near 1, the rest decaying from 0.05) with the Mueller-type two-RDM factors
    two_rdm_h = n_p n_q, two_rdm_x = sqrt(n_p n_q) over the 2 ns spin orbitals, and optionally
    small random pair terms (pair_of, two_rdm_l1, two_rdm_l2)."""
    rng = np.random.default_rng(seed)
    B = ri_tensor(ns, naux, seed, box=box)
    B *= 2.4 / max(1e-30, np.sqrt(np.abs(B).max() * np.sqrt(naux)))
    q = random_orthogonal(ns, rng)
    Bmo = np.einsum("ai,Pab,bj->Pij", q, B.reshape(naux, ns, ns), q, optimize=True).reshape(naux, ns * ns)
    nocc = max(1, ns // 4) if nocc is None else nocc
    e = np.sort(np.concatenate([-3.0 + rng.random(nocc), 0.5 + 3 * rng.random(ns - nocc)]))
    qq = random_orthogonal(ns, rng)
    h = (qq * e) @ qq.T
    occ_sp = np.concatenate([0.97 - 0.05 * rng.random(nocc), 0.05 * np.exp(-np.arange(ns - nocc) / 2.0)])
    occ = np.concatenate([occ_sp, occ_sp])
    out = dict(ns=ns, naux=naux, Bmo=Bmo, h=h, occupations=occ, two_rdm_h=np.outer(occ, occ),
               two_rdm_x=np.sqrt(np.outer(occ, occ)))
    if with_pairs:
        d = 2 * ns
        out["pair_of"] = np.array([(i + 1) % d if i % 2 == 0 else i - 1 for i in range(d)])
        out["two_rdm_l1"] = 0.01 * rng.standard_normal((d, d))
        out["two_rdm_l2"] = 0.01 * rng.standard_normal((d, d))
    return out


def functional_system_complex(n: int, naux: int, seed: int, nocc: int | None = None, with_pairs: bool = False,
                              n_negative: int = 0, box: float = 8.0) -> dict:
    """Fixed-occupation functional-stage inputs for the complex spinor RI tensor (RiMoEri): the
    cube/Gaussian recipe's tensor in a random unitary basis (every B^P Hermitian), a Hermitian h with
    nocc low levels (not diagonal in that basis), spinor occupations (nocc near 1, the rest decaying
    from 0.05) with two_rdm_h = n_p n_q, two_rdm_x = sqrt(n_p n_q), optionally small random pair terms,
    and optionally n_negative leading spinors of a negative-energy branch (levels near -40, empty)."""
    rng = np.random.default_rng(seed)
    B = ri_tensor(n, naux, seed, box=box)
    B *= 2.4 / max(1e-30, np.sqrt(np.abs(B).max() * np.sqrt(naux)))
    u = random_unitary(n, rng)
    Bmo = np.einsum("ai,Pab,bj->Pij", u.conj(), B.reshape(naux, n, n), u, optimize=True).reshape(naux, n * n)
    npos = n - n_negative
    nocc = max(1, npos // 4) if nocc is None else nocc
    e = np.sort(np.concatenate([-3.0 + rng.random(nocc), 0.5 + 3 * rng.random(npos - nocc)]))
    e = np.concatenate([-40.0 - rng.random(n_negative), e])
    uu = random_unitary(n, rng)
    # keep the negative branch on its own block of the spinor space so it stays separable
    if n_negative:
        uu[:n_negative, n_negative:] = 0.0
        uu[n_negative:, :n_negative] = 0.0
        uu[:n_negative, :n_negative] = random_unitary(n_negative, rng)
        uu[n_negative:, n_negative:] = random_unitary(npos, rng)
    h = (uu * e) @ uu.conj().T
    h = 0.5 * (h + h.conj().T)
    occ = np.concatenate([np.zeros(n_negative), 0.97 - 0.05 * rng.random(nocc),
                          0.05 * np.exp(-np.arange(npos - nocc) / 2.0)])
    out = dict(n=n, naux=naux, Bmo=Bmo, h=h, occupations=occ, two_rdm_h=np.outer(occ, occ),
               two_rdm_x=np.sqrt(np.outer(occ, occ)), n_negative=n_negative)
    if with_pairs:
        out["pair_of"] = np.array([(i + 1) % n if i % 2 == 0 else i - 1 for i in range(n)])
        out["two_rdm_l1"] = 0.01 * rng.standard_normal((n, n))
        out["two_rdm_l2"] = 0.01 * rng.standard_normal((n, n))
    return out
