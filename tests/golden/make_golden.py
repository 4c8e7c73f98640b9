"""Generates the golden fixtures in this directory from the REFERENCE ITSELF.

Every output array in ``*.npz`` here was computed by the reference's own RI sources, compiled
unmodified into ``oracle/_ref/librrref.so`` (``make -C oracle``), on seeded synthetic inputs
from ``rerdmft_b200.synth``.  The fixtures pin the numpy restatement (``oracle/ri_oracle.py``)
and the CUDA path; they travel with the repository, so tests on a machine without the
reference tree still compare against the reference's numbers.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py ri_setup   # only ri_setup.npz (the device set-up path)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402
from rerdmft_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent


def save(name, **arrays):
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    print(f"  {name}.npz")


def aux_metric_stand_in(naux, seed):
    """A Gaussian-overlap stand-in for the aux metric (P|Q) (the real one needs libcint): exp(-|r_P -
    r_Q|^2 / 2) over seeded centres, two of them coincident, so the canonical orthogonalisation drops
    one direction as LOWGEN does for a near-dependent aux basis."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, 6.0, size=(naux, 3))
    r[1] = r[0]
    d2 = ((r[:, None, :] - r[None, :, :]) ** 2).sum(-1)
    return np.exp(-0.5 * d2)


def make_setup():
    """The device set-up path: canonical orthogonalisation with its report (LinearAlgebra.cpp:267, :312),
    the metric contraction (ThreeCenterIntegrals.cpp:219-236: restated, since the reference function
    runs only after libcint integrals) and the AO-leg transform (ThreeCenterIntegrals.cpp:191-217,
    the reference's own function)."""
    ref.set_threads(4)
    n_ao, naux_raw, n_out = 10, 60, 8
    M = aux_metric_stand_in(naux_raw, 31)
    Xm, rep = ref.canonical_orth_report(M, 1e-10)
    raw = synth.ri_tensor(n_ao, naux_raw, 32, box=6.0)
    B = Xm.T @ raw
    rng = np.random.default_rng(33)
    t = rng.standard_normal((n_ao, n_out))
    B_legs = ref.transform_ao_legs(B, n_ao, t)
    k = synth.rkb_system(8, 14, 40, 4, seed=23)
    Xh, reph = ref.canonical_orth_report(k["s_full"], 1e-10)
    Sfull = synth.nonrel_system(12, 30, 3, seed=34)["S"]
    Xf, repf = ref.canonical_orth_report(Sfull, 1e-10)
    save("ri_setup", metric=M, metric_x=Xm, metric_report=np.array([rep["n_kept"], rep["n_dropped"],
                                                                     rep["smallest_kept"], rep["largest_dropped"]]),
         raw=raw, B=B, t=t, B_legs=B_legs, s_full=k["s_full"], XXh=Xh @ Xh.conj().T,
         s_full_report=np.array([reph["n_kept"], reph["n_dropped"], reph["smallest_kept"], reph["largest_dropped"]]),
         S_full_rank=Sfull, X_full_rank=Xf)


def main():
    if sys.argv[1:] == ["ri_setup"]:
        return make_setup()
    ref.set_threads(4)
    # --- nonrelativistic Fock builds (NonRelFockMatrixRi.cpp:71) ---
    for n, naux, nocc, seed in [(1, 3, 1, 11), (7, 20, 2, 12), (13, 37, 3, 13), (24, 129, 5, 14), (33, 70, 7, 15)]:
        s = synth.nonrel_system(n, naux, nocc, seed=seed)
        rng = np.random.default_rng(seed + 100)
        # a DIIS-like, non-idempotent density too (the reference's recovery keeps eigenvalues > 0.5)
        c1, _ = synth.occupied_density(n, nocc, rng)
        D_mix = 0.7 * s["D0"] + 0.3 * 2.0 * (s["X"] @ (s["X"].T @ (c1 @ c1.T)))[:, :]
        D_mix = 0.5 * (D_mix + D_mix.T)
        F0 = ref.nonrel_fock(s["h"], s["B"], s["D0"], s["S"], s["X"])
        F1 = ref.nonrel_fock(s["h"], s["B"], D_mix, s["S"], s["X"])
        save(f"nonrel_fock_n{n}_naux{naux}", B=s["B"], h=s["h"], S=s["S"], X=s["X"], D=s["D0"], F=F0, D_mix=D_mix,
             F_mix=F1)
    # rectangular X (a dropped near-linear dependency, LinearAlgebra.cpp:267 with threshold)
    n, naux, nocc = 12, 40, 3
    s = synth.nonrel_system(n, naux, nocc, seed=21)
    S = s["S"].copy()
    v = np.zeros(n)
    v[0], v[1] = 1.0, -1.0
    S = S + 0.0  # make functions 0 and 1 nearly dependent
    S[0, :] = S[1, :] = 0.5 * (S[0, :] + S[1, :])
    S[:, 0] = S[:, 1] = 0.5 * (S[:, 0] + S[:, 1])
    S[0, 0] += 1e-7
    S[1, 1] += 1e-7
    X = ref.canonical_orth(S, 1e-6)
    w, y = np.linalg.eigh(X.T @ s["h"] @ X)
    C = X @ y
    D = 2.0 * C[:, :nocc] @ C[:, :nocc].T
    F = ref.nonrel_fock(s["h"], s["B"], D, S, X)
    save("nonrel_fock_rect", B=s["B"], h=s["h"], S=S, X=X, D=D, F=F)

    # --- X2C Fock builds (X2C_FockMatrixRi.cpp:79) ---
    for nl, naux, ne, seed in [(3, 10, 2, 31), (7, 30, 4, 32), (12, 48, 6, 33)]:
        x = synth.x2c_system(nl, naux, ne, seed=seed)
        F = ref.x2c_fock(x["h"], x["B"], x["P0"], x["S"], x["X"])
        save(f"x2c_fock_nl{nl}_naux{naux}", B=x["B"], h=x["h"], S=x["S"], X=x["X"], P=x["P0"], F=F)

    # --- 4c: riFockTwoElectronDirect and rkbFockMatrix (UkbFockMatrixRi.cpp:35, :185) ---
    for nl, ns, naux, ne, seed in [(3, 5, 14, 2, 41), (5, 9, 33, 4, 42)]:
        k = synth.rkb_system(nl, ns, naux, ne, seed=seed)
        F = ref.rkb_fock(k["h"], nl, ns, k["B_LL"], k["B_SS"], k["v_total"], k["s_full"], k["x_full"], k["P0"])
        rng = np.random.default_rng(seed)
        nu = 2 * nl + 2 * ns
        c_occ = synth.random_unitary(nu, rng)[:, :ne] * 0.7
        occ = 0.6 + 0.4 * rng.random(ne)
        p_ukb = (c_occ * occ) @ c_occ.conj().T
        G = ref.ukb_two_electron(nl, ns, k["B_LL"], k["B_SS"], p_ukb, c_occ, occ)
        save(f"rkb_fock_nl{nl}_ns{ns}", B_LL=k["B_LL"], B_SS=k["B_SS"], v_total=k["v_total"], s_full=k["s_full"],
             x_full=k["x_full"], h=k["h"], P=k["P0"], F=F, P_ukb=p_ukb, C_occ=c_occ, occ=occ, G=G)

    # --- MO transforms (NonRelSpinRiMoEri.cpp:13/:45, RiMoEri.cpp:64/:88/:112) ---
    rng = np.random.default_rng(51)
    n, naux = 9, 25
    B = synth.ri_tensor(n, naux, 51, box=6.0)
    C = synth.random_orthogonal(n, rng)
    Bmo = ref.nonrel_mo_build(B, C)
    U = np.kron(np.eye(2), synth.random_orthogonal(n, rng))
    U[n:, n:] += 1e-5 * rng.standard_normal((n, n))  # within the 1e-3 alpha/beta tolerance
    Brot = ref.nonrel_mo_rotated(Bmo, n, U)
    emb = ref.nonrel_mo_embedded(Bmo, n)
    quads = rng.integers(0, 2 * n, (64, 4))
    eri = ref.nonrel_mo_eri(Bmo, n, quads)
    save("nonrel_mo", B=B, C=C, Bmo=Bmo, U=U, Brot=Brot, emb=emb, quads=quads, eri=eri)

    nl, ns, naux = 4, 6, 18
    B_LL = synth.ri_tensor(nl, naux, 52, box=6.0)
    B_SS = synth.ri_tensor(ns, naux, 53, box=6.0)
    nt = 12
    c_ukb = synth.random_unitary(2 * nl + 2 * ns, rng)[:, :nt]
    Bc = ref.ri_mo_build(nl, ns, B_LL, B_SS, c_ukb)
    Uc = synth.random_unitary(nt, rng)
    Bcr = ref.ri_mo_rotated(Bc, nt, Uc)
    Bpos = ref.ri_mo_positive(Bc, nt, 4)
    quads = rng.integers(0, nt, (64, 4))
    eric = ref.ri_mo_eri(Bc, nt, quads)
    save("ri_mo", B_LL=B_LL, B_SS=B_SS, c_ukb=c_ukb, Bmo=Bc, U=Uc, Brot=Bcr, Bpos=Bpos, quads=quads, eri=eric)

    # --- generalized Fock (RiGemmFock.cpp:52 riHxFockGemm, both overloads) ---
    n = nt
    hc = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    occ = rng.random(n)
    h2, x2, l1, l2 = (rng.standard_normal((n, n)) for _ in range(4))
    po = np.arange(n) ^ 1
    Fc = ref.hx_fock_complex(Bc, n, hc, occ, h2, x2, po, l1, l2)
    Fc0 = ref.hx_fock_complex(Bc, n, hc, occ, h2, x2)
    nsp = 9
    n = 2 * nsp
    hr = rng.standard_normal((n, n))
    occr = rng.random(n)
    h2r, x2r, l1r, l2r = (rng.standard_normal((n, n)) for _ in range(4))
    por = (np.arange(n) + nsp) % n
    Fr = ref.hx_fock_nonrel(Bmo, nsp, hr, occr, h2r, x2r, por, l1r, l2r)
    save("hx_fock", Bc=Bc, hc=hc, occ=occ, h2=h2, x2=x2, l1=l1, l2=l2, po=po, Fc=Fc, Fc0=Fc0, Bmo=Bmo, hr=hr,
         occr=occr, h2r=h2r, x2r=x2r, l1r=l1r, l2r=l2r, por=por, Fr=Fr)

    # --- DIIS (DIIS.cpp:53, :79) ---
    E = rng.standard_normal((9, 40))
    V = rng.standard_normal((9, 40))
    E[6] = E[5] * (1 + 1e-16)  # a singular step: the oldest pairs get dropped
    out, wc = ref.diis_sequence(5, E, V)
    Ec = rng.standard_normal((7, 30)) + 1j * rng.standard_normal((7, 30))
    Vc = rng.standard_normal((7, 30)) + 1j * rng.standard_normal((7, 30))
    outc, wcc = ref.diis_sequence(4, Ec, Vc)
    Fm, Pm, Sm = (rng.standard_normal((8, 8)) for _ in range(3))
    comm = ref.commutator_error(Fm, Pm, Sm)
    save("diis", E=E, V=V, out=out, wc=wc, Ec=Ec, Vc=Vc, outc=outc, wcc=wcc, Fm=Fm, Pm=Pm, Sm=Sm, comm=comm)

    # --- SCF loops (NonRelHartreeFock.cpp:117, X2C_HF.cpp:43, C4_DHF.cpp:45) ---
    s = synth.nonrel_system(16, 60, 4, seed=61)
    r = ref.nonrel_scf(s)
    save("scf_nonrel", B=s["B"], h=s["h"], S=s["S"], X=s["X"], D0=s["D0"], n_electrons=s["n_electrons"],
         energy=r["energy"], iterations=r["iterations"], history=r["history"], P=r["P"])
    x = synth.x2c_system(8, 32, 4, seed=62)
    r = ref.x2c_scf(x)
    save("scf_x2c", B=x["B"], h=x["h"], S=x["S"], X=x["X"], P0=x["P0"], n_electrons=x["n_electrons"],
         energy=r["energy"], iterations=r["iterations"], history=r["history"], P=r["P"])
    k = synth.rkb_system(4, 7, 24, 4, seed=63)
    r = ref.dhf_scf(k)
    save("scf_dhf", B_LL=k["B_LL"], B_SS=k["B_SS"], v_total=k["v_total"], s_full=k["s_full"], x_full=k["x_full"],
         h=k["h"], P0=k["P0"], n_electrons=k["n_electrons"], nl=k["nl"], ns=k["ns"], energy=r["energy"],
         iterations=r["iterations"], history=r["history"], P=r["P"])

    # --- canonical orthogonalisation (LinearAlgebra.cpp:267, :312) ---
    Xs = ref.canonical_orth(S, 1e-6)
    Xh = ref.canonical_orth(k["s_full"], 1e-10)
    save("orth", S=S, X=Xs, s_full=k["s_full"], XXh=Xh @ Xh.conj().T)
    make_setup()


if __name__ == "__main__":
    main()
