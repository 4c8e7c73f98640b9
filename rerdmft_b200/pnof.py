"""PNOF / GNOF functionals of the functional stage over the device MO tensors, and their full
optimisation (orbitals by the device ADAM, occupations on the host from the device J/K).

* ``nonrel_geminals``       the coupled-subspace partition of a closed-shell NON_REL reference in the
                            spin-orbital index space of RiNonRelSpinMoEri (i = spatial orbital, ibar = i + n):
                            subspace k anchored on HOMO-k with the next (coupling-1) virtual pairs
                            (src/Occ_opt/Orb_subspaces.h, buildPnofGeminals PNOFs.cpp:158)
* ``occupations_from_gammas`` the cos^2 / sin^2 stick-breaking angles of one subspace
                            (pnofSubspaceOccupationsFromGammas, PNOFs.cpp:814)
* ``pi_pair``               Pi^intra / Pi^inter of PNOF5, PNOF7, PNOF7s and GNOF (PNOFs.cpp:36-206)
* ``full_two_rdm``          the actual-orbital two_rdm_h / x / l1 / l2 and pair_of that the generalized Fock
                            and the rotation problem take (buildPnofFullTwoRdm, PnofFock.cpp:29-139)
* ``electronic_energy``     the geminal form of the energy from h_ii, J_ij, K_ij
                            (pnofElectronicEnergy, PNOFs.cpp:271-330, non-relativistic)
* ``optimize_occupations``  the occupations at fixed orbitals: L-BFGS over the gamma angles (the
                            reference's unconstrained route, FullOptimization.cpp:970-1010)
* ``run_pnof_optimization`` the FULL_OPTIMIZATION macro loop (FullOptimization.cpp:2691-2915): an ADAM
                            orbital run, then the occupations at the new orbitals, until the energy
                            changes by less than `tol` without a restart request
"""
from __future__ import annotations

import math
import time

import numpy as np

FUNCTIONALS = {"PNOF5": 0, "PNOF7": 1, "PNOF7S": 2, "GNOF": 3}


def nonrel_geminals(n_spatial: int, n_occ_pairs: int, coupling: int, n_subspaces: int | None = None) -> np.ndarray:
    """Geminals (rows i, ibar, subspace_id, is_principal) of a closed-shell NON_REL reference with the
    lowest `n_occ_pairs` spatial orbitals occupied: the occupied pairs below the `n_subspaces` frontier
    ones are frozen (their own trivial subspaces, occupation 1), subspace k is anchored on HOMO-k and
    owns the k-th block of (coupling - 1) virtual pairs above the Fermi level; virtual pairs beyond the
    blocks are not geminals (occupation 0).  Spin-orbital indices: alpha i, beta i + n_spatial."""
    n_sub = n_occ_pairs if n_subspaces is None else n_subspaces
    if coupling < 2 or not (1 <= n_sub <= n_occ_pairs):
        raise ValueError("nonrel_geminals: coupling >= 2 and 1 <= n_subspaces <= n_occ_pairs")
    if n_occ_pairs + n_sub * (coupling - 1) > n_spatial:
        raise ValueError("nonrel_geminals: not enough virtual orbitals for the coupling")
    rows, sid = [], 0
    for i in range(n_occ_pairs - n_sub):  # frozen core
        rows.append((i, i + n_spatial, sid, 1))
        sid += 1
    for k in range(n_sub):
        p = n_occ_pairs - 1 - k
        rows.append((p, p + n_spatial, sid, 1))
        for v in range(coupling - 1):
            q = n_occ_pairs + k * (coupling - 1) + v
            rows.append((q, q + n_spatial, sid, 0))
        sid += 1
    return np.array(rows, dtype=np.int64)


def occupations_from_gammas(coupling: int, gammas) -> np.ndarray:
    """Occupations of one subspace (principal first) from its coupling - 1 angles: n_0 = 1/2 + 1/2 cos^2 g_0,
    then each virtual takes sin^2 g_k of what is left and the last virtual the rest."""
    g = np.asarray(gammas, dtype=float)
    occ = np.empty(coupling)
    occ[0] = 0.5 + 0.5 * math.cos(g[0]) ** 2
    rest = 1.0 - occ[0]
    for k in range(coupling - 2):
        occ[1 + k] = rest * math.sin(g[k + 1]) ** 2
        rest -= occ[1 + k]
    occ[coupling - 1] = rest
    return occ


def occupations_of(geminals: np.ndarray, coupling: int, gammas, n_total: int) -> np.ndarray:
    """Spin-orbital occupations (n_i = n_ibar) from the angles of every coupled subspace (in subspace
    order); frozen geminals get 1, orbitals of no geminal 0."""
    occ = np.zeros(n_total)
    per = coupling - 1
    s = 0
    for sid in np.unique(geminals[:, 2]):
        rows = geminals[geminals[:, 2] == sid]
        if len(rows) == 1:
            occ[rows[0, 0]] = occ[rows[0, 1]] = 1.0
            continue
        o = occupations_from_gammas(coupling, gammas[s * per:(s + 1) * per])
        for v, r in enumerate(rows):
            occ[r[0]] = occ[r[1]] = o[v]
        s += 1
    return occ


def _gnof_occ_d(n_i: float, h_principal: float) -> float:
    """GNOF's dynamic occupation n_i^d = n_i exp(-(h_p / (0.02 sqrt 2))^2)."""
    r = h_principal / (0.02 * math.sqrt(2.0))
    return n_i * math.exp(-r * r)


def pi_pair(functional: int, geminals: np.ndarray, occ: np.ndarray, a: int, b: int, principal_occ: dict) -> float:
    """Pi_ab of two distinct geminals: intra-subspace -+sqrt(n_a n_b) (minus when one is a principal);
    inter-subspace 0 (PNOF5), -sqrt(n_a n_b h_a h_b) (PNOF7), -4 n_a n_b h_a h_b (PNOF7s), or GNOF's
    n^d_a n^d_b - sqrt(n_a n_b h_a h_b) -+ sqrt(n^d_a n^d_b) (minus for a principal / virtual pair,
    0 between two principals)."""
    ga, gb = geminals[a], geminals[b]
    n_a, n_b = occ[ga[0]], occ[gb[0]]
    if ga[2] == gb[2]:
        s = math.sqrt(n_a * n_b)
        return -s if (ga[3] or gb[3]) else s
    h_a, h_b = 1.0 - n_a, 1.0 - n_b
    if functional == 0:
        return 0.0
    if functional == 1:
        return -math.sqrt(n_a * n_b * h_a * h_b)
    if functional == 2:
        return -4.0 * n_a * n_b * h_a * h_b
    if ga[3] and gb[3]:
        return 0.0
    nd_a = _gnof_occ_d(n_a, 1.0 - principal_occ[ga[2]])
    nd_b = _gnof_occ_d(n_b, 1.0 - principal_occ[gb[2]])
    base = nd_a * nd_b - math.sqrt(n_a * n_b * h_a * h_b)
    cross = math.sqrt(nd_a * nd_b)
    return base - cross if bool(ga[3]) != bool(gb[3]) else base + cross


def _principal_occ(geminals, occ):
    return {int(g[2]): occ[g[0]] for g in geminals if g[3]}


def full_two_rdm(functional: int, geminals: np.ndarray, occ: np.ndarray, n_total: int) -> dict:
    """two_rdm_h / x / l1 / l2 (n_total x n_total) and pair_of for the generalized Fock: within a geminal
    (i, ibar) both h and x are n_a; between geminals a, b every member combination gets
    n_a n_b - Delta_ab (Delta = n_a n_b inside one subspace) in h and x, and the pair term +-Pi_ab / 4
    in l1 (plus for matching bar parity) with l2 = -l1."""
    h2 = np.zeros((n_total, n_total))
    x2 = np.zeros((n_total, n_total))
    l1 = np.zeros((n_total, n_total))
    pocc = _principal_occ(geminals, occ)
    for a, ga in enumerate(geminals):
        i, ib = int(ga[0]), int(ga[1])
        n_a = occ[i]
        h2[i, ib] = h2[ib, i] = x2[i, ib] = x2[ib, i] = n_a
        for b in range(a + 1, len(geminals)):
            gb = geminals[b]
            n_b = occ[gb[0]]
            hx = n_a * n_b - (n_a * n_b if ga[2] == gb[2] else 0.0)
            pi = pi_pair(functional, geminals, occ, a, b, pocc)
            for pp, P in enumerate((i, ib)):
                for qq, Q in enumerate((int(gb[0]), int(gb[1]))):
                    h2[P, Q] = h2[Q, P] = x2[P, Q] = x2[Q, P] = hx
                    l1[P, Q] = l1[Q, P] = pi / 4.0 if pp == qq else -pi / 4.0
    pair_of = np.arange(n_total, dtype=np.int64)
    for g in geminals:
        pair_of[g[0]], pair_of[g[1]] = g[1], g[0]
    return dict(two_rdm_h=h2, two_rdm_x=x2, two_rdm_l1=l1, two_rdm_l2=-l1, pair_of=pair_of)


def _pi_matrix(functional: int, geminals: np.ndarray, occ: np.ndarray) -> np.ndarray:
    """Pi_ab of every pair of distinct geminals at once (the rules of pi_pair; diagonal 0)."""
    ng = len(geminals)
    n = occ[geminals[:, 0]]
    sub = geminals[:, 2]
    prin = geminals[:, 3].astype(bool)
    same = sub[:, None] == sub[None, :]
    nn = np.outer(n, n)
    hh = np.outer(1.0 - n, 1.0 - n)
    intra = np.where(prin[:, None] | prin[None, :], -np.sqrt(nn), np.sqrt(nn))
    if functional == 0:
        inter = np.zeros((ng, ng))
    elif functional == 1:
        inter = -np.sqrt(nn * hh)
    elif functional == 2:
        inter = -4.0 * nn * hh
    else:
        pocc = _principal_occ(geminals, occ)
        hp = np.array([1.0 - pocc[int(s_)] for s_ in sub])
        nd = n * np.exp(-(hp / (0.02 * math.sqrt(2.0))) ** 2)
        base = np.outer(nd, nd) - np.sqrt(nn * hh)
        cross = np.sqrt(np.outer(nd, nd))
        mixed = prin[:, None] != prin[None, :]
        inter = np.where(mixed, base - cross, base + cross)
        inter[prin[:, None] & prin[None, :]] = 0.0
    pi = np.where(same, intra, inter)
    np.fill_diagonal(pi, 0.0)
    return pi


def electronic_energy(functional: int, geminals: np.ndarray, occ: np.ndarray, h_diag, J, K) -> float:
    """Non-relativistic PNOF energy from the actual-orbital h_pp (spin orbitals) and the representative
    J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i): sum_p n_p h_pp + sum_ab [h_ab J_ab - x_ab K_ab]
    + sum_{a != b} Pi_ab K_ab over geminals a, b, with h_aa = n_a, x_aa = 0, h_ab = 2 (n_a n_b - Delta_ab),
    x_ab = n_a n_b - Delta_ab (Delta = n_a n_b inside one subspace)."""
    h_diag = np.asarray(h_diag)
    reps = geminals[:, 0]
    n = occ[reps]
    e = float(np.sum(occ[geminals[:, 0]] * h_diag[geminals[:, 0]] + occ[geminals[:, 1]] * h_diag[geminals[:, 1]]))
    Jr = np.asarray(J)[np.ix_(reps, reps)]
    Kr = np.asarray(K)[np.ix_(reps, reps)]
    same = geminals[:, 2][:, None] == geminals[:, 2][None, :]
    hx = np.where(same, 0.0, np.outer(n, n))
    np.fill_diagonal(hx, 0.0)
    e += float(np.sum(n * np.diag(Jr)))
    e += float(np.sum(2.0 * hx * Jr - hx * Kr))
    e += float(np.sum(_pi_matrix(functional, geminals, occ) * Kr))
    return e


def optimize_occupations(functional: int, geminals: np.ndarray, coupling: int, h_diag, J, K, gammas0,
                         n_total: int, gtol: float = 1e-10) -> dict:
    """Occupations at fixed orbitals: L-BFGS over the coupled subspaces' gamma angles (every angle gives
    a feasible occupation set), central-difference gradient; returns the angles, occupations, energy."""
    from scipy.optimize import minimize

    g0 = np.asarray(gammas0, dtype=float)
    if g0.size == 0:
        occ = occupations_of(geminals, coupling, g0, n_total)
        return dict(gammas=g0, occupations=occ, energy=electronic_energy(functional, geminals, occ, h_diag, J, K),
                    iterations=0, converged=True)

    def f(g):
        return electronic_energy(functional, geminals, occupations_of(geminals, coupling, g, n_total), h_diag, J, K)

    def grad(g):
        out = np.empty_like(g)
        for k in range(g.size):
            d = np.zeros_like(g)
            d[k] = 1e-6
            out[k] = (f(g + d) - f(g - d)) / 2e-6
        return out

    r = minimize(f, g0, jac=grad, method="L-BFGS-B", options=dict(gtol=gtol, ftol=1e-15, maxiter=500))
    occ = occupations_of(geminals, coupling, r.x, n_total)
    return dict(gammas=r.x, occupations=occ, energy=float(r.fun), iterations=int(r.nit), converged=bool(r.success))


def run_pnof_optimization(problem, functional: str, geminals: np.ndarray, coupling: int, tol: float = 1e-8,
                          max_macro: int = 200, preconditioner=None, clip: float = 16.0, quantile: float = 0.9,
                          polish: bool = True) -> dict:
    """FULL_OPTIMIZATION of a PNOF functional on `problem` (orbopt.RotationProblem over the spin-orbital
    tensor): occupations first at the starting orbitals, then macro-iterations of one ADAM orbital run
    (scales from `preconditioner` before each run while it is in use, plain ADAM after, as
    orbopt.run_full_optimization) and the occupations at the new orbitals, until two successive energies
    differ by less than `tol` and ADAM asked for no restart."""
    from . import orbopt

    f = FUNCTIONALS[functional.upper()]
    n_total = problem.d
    n_sub = sum(1 for s in np.unique(geminals[:, 2]) if (geminals[:, 2] == s).sum() > 1)
    gam = np.full(n_sub * (coupling - 1), math.pi / 4.0)  # the reference's default guess
    t0 = time.perf_counter()

    def occ_step(g):
        J, K, hd = problem.jk_and_h_diag()
        return optimize_occupations(f, geminals, coupling, hd, J, K, g, n_total)

    res = occ_step(gam)
    gam = res["gammas"]
    problem.set_functional(res["occupations"], **full_two_rdm(f, geminals, res["occupations"], n_total))
    e_prev = res["energy"]
    history, steps, m, scaled_macro = [e_prev], 0, 0, 0
    converged = False
    phases = ["scaled", "plain"] if (preconditioner is not None and polish) else (
        ["scaled"] if preconditioner is not None else ["plain"])
    for phase in phases:
        if phase == "plain":
            problem.set_scales(None)
        converged = False
        while m < max_macro:
            m += 1
            if phase == "scaled":
                scaled_macro += 1
                problem.set_scales(preconditioner.scales(problem, clip, quantile=quantile))
            r = problem.run()
            steps += r["iterations"]
            res = occ_step(gam)
            gam = res["gammas"]
            problem.set_functional(res["occupations"], **full_two_rdm(f, geminals, res["occupations"], n_total))
            e = res["energy"]
            history.append(e)
            if abs(e - e_prev) < tol and not r["restart_requested"]:
                converged = True
                e_prev = e
                break
            e_prev = e
    return dict(macro_iterations=m, adam_steps=steps, energy=e_prev, converged=converged, occupations=res["occupations"],
                gammas=gam, scaled_macro_iterations=scaled_macro, seconds=time.perf_counter() - t0,
                history=np.array(history))
