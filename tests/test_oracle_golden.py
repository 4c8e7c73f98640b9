"""Pins the numpy restatement (oracle/ri_oracle.py) to golden outputs of the reference itself."""
import numpy as np
import pytest

from conftest import GOLDEN, golden
from oracle import ri_oracle as o

TOL = 1e-12


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("nonrel_fock_*.npz")))
def test_nonrel_fock(name):
    g = golden(name)
    F = o.nonrel_fock(g["h"], g["B"], g["D"], g["S"], g["X"])
    assert np.abs(F - g["F"]).max() < TOL
    if "D_mix" in g:
        assert np.abs(o.nonrel_fock(g["h"], g["B"], g["D_mix"], g["S"], g["X"]) - g["F_mix"]).max() < TOL


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("x2c_fock_*.npz")))
def test_x2c_fock(name):
    g = golden(name)
    F = o.x2c_fock(g["h"], g["B"], g["P"], g["S"], g["X"])
    assert np.abs(F - g["F"]).max() < TOL


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("rkb_fock_*.npz")))
def test_rkb_and_ukb(name):
    g = golden(name)
    nl, ns = g["B_LL"].shape[1] ** 0.5, g["B_SS"].shape[1] ** 0.5
    nl, ns = int(round(nl)), int(round(ns))
    F = o.rkb_fock(g["h"], nl, ns, g["B_LL"], g["B_SS"], g["v_total"], g["s_full"], g["x_full"], g["P"])
    assert np.abs(F - g["F"]).max() < 1e-11
    G = o.ukb_two_electron(nl, ns, g["B_LL"], g["B_SS"], g["P_ukb"], g["C_occ"], g["occ"])
    assert np.abs(G - g["G"]).max() < TOL


def test_nonrel_mo():
    g = golden("nonrel_mo")
    n = g["C"].shape[0]
    assert np.abs(o.nonrel_mo_build(g["B"], g["C"]) - g["Bmo"]).max() < TOL
    assert np.abs(o.nonrel_mo_rotated(g["Bmo"], n, g["U"]) - g["Brot"]).max() < TOL
    assert np.abs(o.nonrel_mo_embedded(g["Bmo"], n) - g["emb"]).max() == 0.0
    assert np.abs(o.nonrel_mo_eri(g["Bmo"], n, g["quads"]) - g["eri"]).max() < TOL
    bad = g["U"].copy()
    bad[0, n] = 0.01
    with pytest.raises(ValueError):
        o.nonrel_mo_rotated(g["Bmo"], n, bad)


def test_ri_mo():
    g = golden("ri_mo")
    nl, ns = int(round(g["B_LL"].shape[1] ** 0.5)), int(round(g["B_SS"].shape[1] ** 0.5))
    nt = g["c_ukb"].shape[1]
    assert np.abs(o.ri_mo_build(nl, ns, g["B_LL"], g["B_SS"], g["c_ukb"]) - g["Bmo"]).max() < TOL
    assert np.abs(o.ri_mo_rotated(g["Bmo"], nt, g["U"]) - g["Brot"]).max() < TOL
    assert np.abs(o.ri_mo_positive(g["Bmo"], nt, 4) - g["Bpos"]).max() == 0.0
    assert np.abs(o.ri_mo_eri(g["Bmo"], nt, g["quads"]) - g["eri"]).max() < TOL


def test_jkl_matches_element_access():
    g = golden("ri_mo")
    nt = g["c_ukb"].shape[1]
    po = np.arange(nt) ^ 1
    J, K, Lm = o.jkl_matrices(g["Bmo"], nt, po)
    for i in range(nt):
        for j in range(nt):
            q = np.array([[i, j, i, j], [i, j, j, i], [po[i], j, j, po[i]]])
            e = o.ri_mo_eri(g["Bmo"], nt, q)
            assert abs(J[i, j] - e[0]) < TOL and abs(K[i, j] - e[1]) < TOL and abs(Lm[i, j] - e[2]) < TOL


def test_hx_fock():
    g = golden("hx_fock")
    Fc = o.hx_fock(g["hc"], g["Bc"], g["occ"], g["h2"], g["x2"], g["po"], g["l1"], g["l2"])
    assert np.abs(Fc - g["Fc"]).max() < TOL
    assert np.abs(o.hx_fock(g["hc"], g["Bc"], g["occ"], g["h2"], g["x2"]) - g["Fc0"]).max() < TOL
    nsp = int(round(g["Bmo"].shape[1] ** 0.5))
    emb = o.nonrel_mo_embedded(g["Bmo"], nsp)
    Fr = o.hx_fock(g["hr"], emb, g["occr"], g["h2r"], g["x2r"], g["por"], g["l1r"], g["l2r"])
    assert np.abs(Fr - g["Fr"]).max() < TOL


def test_diis():
    g = golden("diis")
    d = o.Diis(5)
    for t in range(g["E"].shape[0]):
        r = d.extrapolate(g["E"][t], g["V"][t])
        assert np.abs(r - g["out"][t]).max() < 1e-11
        assert len(d.last_weights) == g["wc"][t]
    d = o.Diis(4)
    for t in range(g["Ec"].shape[0]):
        r = d.extrapolate(g["Ec"][t], g["Vc"][t])
        assert np.abs(r - g["outc"][t]).max() < 1e-11
        assert len(d.last_weights) == g["wcc"][t]
    assert np.abs(o.commutator_error(g["Fm"], g["Pm"], g["Sm"]) - g["comm"]).max() < TOL


def test_scf_loops():
    g = golden("scf_nonrel")
    sysd = dict(B=g["B"], h=g["h"], S=g["S"], X=g["X"], D0=g["D0"], n_electrons=int(g["n_electrons"]))
    r = o.nonrel_scf(sysd)
    assert r["iterations"] == int(g["iterations"])
    assert np.abs(r["history"] - g["history"]).max() < 1e-10
    g = golden("scf_x2c")
    sysd = dict(B=g["B"], h=g["h"], S=g["S"], X=g["X"], P0=g["P0"], n_electrons=int(g["n_electrons"]))
    r = o.x2c_scf(sysd)
    assert r["iterations"] == int(g["iterations"])
    assert np.abs(r["history"] - g["history"]).max() < 1e-10
    g = golden("scf_dhf")
    sysd = {k: g[k] for k in ("B_LL", "B_SS", "v_total", "s_full", "x_full", "h", "P0")}
    sysd.update(nl=int(g["nl"]), ns=int(g["ns"]), n_electrons=int(g["n_electrons"]))
    r = o.dhf_scf(sysd)
    assert r["iterations"] == int(g["iterations"])
    assert np.abs(r["history"] - g["history"]).max() < 1e-10


def test_orthogonalisation():
    g = golden("orth")
    X = o.canonical_orthogonalize(g["S"], 1e-6)
    assert X.shape == g["X"].shape
    assert np.abs(X @ X.T - g["X"] @ g["X"].T).max() < 1e-9
    Xh = o.canonical_orthogonalize_hermitian(g["s_full"], 1e-10)
    assert np.abs(Xh @ Xh.conj().T - g["XXh"]).max() < 1e-10


def test_setup_path_restatements():
    """The numpy restatements of the metric contraction and the AO-leg transform against the fixture
    (the AO legs from the reference's own transformRiThreeCenterAoLegs), and of the canonical
    orthogonalisation against the reference's X and report."""
    g = golden("ri_setup")
    assert np.abs(o.three_center_tensor(g["raw"], g["metric_x"]) - g["B"]).max() < 1e-12
    n_ao = g["t"].shape[0]
    assert np.abs(o.transform_ao_legs(g["B"], n_ao, g["t"]) - g["B_legs"]).max() < 1e-12
    X = o.canonical_orthogonalize(g["metric"], 1e-10)
    assert X.shape == g["metric_x"].shape and int(g["metric_report"][1]) == 1
    assert np.abs(X @ X.T - g["metric_x"] @ g["metric_x"].T).max() < 1e-8
    assert np.abs(o.canonical_orthogonalize(g["S_full_rank"], 1e-10) - g["X_full_rank"]).max() < 1e-12
    Xh = o.canonical_orthogonalize_hermitian(g["s_full"], 1e-10)
    assert np.abs(Xh @ Xh.conj().T - g["XXh"]).max() < 1e-10


def test_complex_rotation_problem_restatement(ref_lib):
    """The complex RotationProblem restatement against the reference's own pieces: its generalized
    Fock and orbitalGradient give the pair gradient, its spinorRotationMatrix the rotation, its
    Adam<complex>::step the steps of the optimiser's first iterations.  Without pair terms (random
    l1 / l2 are not consistent with the trace form of the energy) the gradient is the derivative of
    the energy along the real and imaginary parts of each pair's step."""
    from rerdmft_b200 import synth

    f = synth.functional_system_complex(8, 24, 11, with_pairs=True, n_negative=2)
    args = (f["pair_of"], f["two_rdm_l1"], f["two_rdm_l2"])
    pb = o.RotationProblemComplexNumpy(f["Bmo"], f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"], *args,
                                       n_negative=2)
    assert all(p >= 2 and q >= 2 for p, q in pb.pairs) and len(pb.pairs) == 15
    F = ref_lib.hx_fock_complex(f["Bmo"], 8, f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"], *args)
    assert np.abs(pb.fock() - F).max() <= 1e-12
    G = ref_lib.orbital_gradient(F)
    g = pb.gradient()
    assert np.abs(g - np.array([G[p, q] for p, q in pb.pairs])).max() <= 1e-12
    rng = np.random.default_rng(1)
    step = 0.05 * (rng.standard_normal(len(pb.pairs)) + 1j * rng.standard_normal(len(pb.pairs)))
    k = o.kappa_matrix(8, pb.pairs, step)
    assert np.abs(o.rotation_matrix(k) - ref_lib.rotation_matrix(k)).max() <= 1e-13
    gs = np.stack([g, 0.5 * g, -g])
    ref_steps = ref_lib.adam_steps(gs)
    m1, m2, mx = np.zeros_like(g), np.zeros(g.size), np.zeros(g.size)
    for t in range(1, 4):
        m1 = 0.7 * m1 + 0.3 * gs[t - 1]
        m2 = 0.9 * m2 + 0.1 * (gs[t - 1].real ** 2 + gs[t - 1].imag ** 2)
        mx = np.maximum(mx, m2 / (1 - 0.9 ** t))
        st = -0.01 * (m1 / (1 - 0.7 ** t)) / (np.sqrt(mx) + 1e-15)
        assert np.abs(st - ref_steps[t - 1]).max() <= 1e-15
    f = synth.functional_system_complex(8, 24, 11, n_negative=2)
    pb = o.RotationProblemComplexNumpy(f["Bmo"], f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"],
                                       n_negative=2)
    g = pb.gradient()
    e0, eps = pb.energy(), 1e-6
    for comp in (1.0, 1j):
        d = np.zeros(len(pb.pairs), dtype=complex)
        d[4] = eps * comp
        pb.save_best()
        pb.rotate(d)
        ep = pb.energy()
        pb.restore_best()
        pb.rotate(-d)
        em = pb.energy()
        pb.restore_best()
        want = g[4].real if comp == 1.0 else g[4].imag
        assert abs((ep - em) / (2 * eps) - want) <= 1e-7 * max(1.0, abs(want))
    assert abs(pb.energy() - e0) <= 1e-14
