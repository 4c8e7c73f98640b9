"""Parity of the MO-basis RI path (transforms, rotations, element access, J/K/L, generalized Fock)
with the reference: golden fixtures from the compiled reference and the numpy restatement."""
import numpy as np
import pytest

from conftest import golden
from oracle import ri_oracle as o
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import mo, ri  # noqa: E402
from rerdmft_b200._lib import RrError  # noqa: E402

TOL = 1e-10


def test_nonrel_golden():
    g = golden("nonrel_mo")
    n = g["C"].shape[0]
    src = ri.RiNonRelEriSource(n, g["B"], np.eye(n), np.eye(n))
    m = mo.buildRiNonRelSpinMoEri(src, n, g["C"])
    assert np.abs(m.b() - g["Bmo"]).max() <= TOL
    r = m.rotated(g["U"])
    assert np.abs(r.b() - g["Brot"]).max() <= TOL
    assert np.abs(m.embeddedB() - g["emb"]).max() <= TOL
    assert np.abs(m.eri(g["quads"]) - g["eri"]).max() <= TOL
    assert m.dim0() == 2 * n and m.nSpatial() == n
    bad = g["U"].copy()
    bad[0, n] = 0.01
    with pytest.raises(RrError, match="not spin-restricted"):
        m.rotated(bad)


def test_ukb_golden():
    g = golden("ri_mo")
    nl, ns = int(round(g["B_LL"].shape[1] ** 0.5)), int(round(g["B_SS"].shape[1] ** 0.5))
    src = ri.RiDirectEriSource(nl, ns, g["B_LL"], g["B_SS"])
    m = mo.buildRiMoEri(src, g["c_ukb"])
    assert np.abs(m.b() - g["Bmo"]).max() <= TOL
    nt = g["c_ukb"].shape[1]
    assert np.abs(m.rotated(g["U"]).b() - g["Brot"]).max() <= TOL
    assert np.abs(m.positiveBlock(4).b() - g["Bpos"]).max() <= TOL
    assert np.abs(m.eri(g["quads"]) - g["eri"]).max() <= TOL
    assert m.dim() == nt


@pytest.mark.parametrize("n,naux", [(1, 3), (17, 50), (64, 200), (130, 333)])
def test_nonrel_vs_oracle(n, naux):
    rng = np.random.default_rng(n)
    B = synth.ri_tensor(n, naux, n, box=6.0)
    C = synth.random_orthogonal(n, rng)
    src = ri.RiNonRelEriSource(n, B, np.eye(n), np.eye(n))
    m = mo.buildRiNonRelSpinMoEri(src, n, C)
    ref = o.nonrel_mo_build(B, C)
    assert np.abs(m.b() - ref).max() <= TOL
    U = np.kron(np.eye(2), synth.random_orthogonal(n, rng))
    assert np.abs(m.rotated(U).b() - o.nonrel_mo_rotated(ref, n, U)).max() <= TOL
    po = (np.arange(2 * n) + n) % (2 * n)
    J, K, Lm = m.jkl(po)
    quads = np.array([[i, j, i, j] for i in range(2 * n) for j in range(2 * n)])
    Je = o.nonrel_mo_eri(ref, n, quads).reshape(2 * n, 2 * n)
    quads = np.array([[i, j, j, i] for i in range(2 * n) for j in range(2 * n)])
    Ke = o.nonrel_mo_eri(ref, n, quads).reshape(2 * n, 2 * n)
    quads = np.array([[po[i], j, j, po[i]] for i in range(2 * n) for j in range(2 * n)])
    Le = o.nonrel_mo_eri(ref, n, quads).reshape(2 * n, 2 * n)
    assert np.abs(J - Je).max() <= TOL and np.abs(K - Ke).max() <= TOL and np.abs(Lm - Le).max() <= TOL


@pytest.mark.parametrize("nl,ns,naux,nt", [(3, 5, 11, 7), (10, 20, 60, 24), (25, 40, 100, 60)])
def test_ukb_vs_oracle(nl, ns, naux, nt):
    rng = np.random.default_rng(nl)
    B_LL = synth.ri_tensor(nl, naux, nl, box=6.0)
    B_SS = synth.ri_tensor(ns, naux, ns, box=6.0)
    c = synth.random_unitary(2 * nl + 2 * ns, rng)[:, :nt]
    src = ri.RiDirectEriSource(nl, ns, B_LL, B_SS)
    m = mo.buildRiMoEri(src, c)
    ref = o.ri_mo_build(nl, ns, B_LL, B_SS, c)
    assert np.abs(m.b() - ref).max() <= TOL
    U = synth.random_unitary(nt, rng)
    assert np.abs(m.rotated(U).b() - o.ri_mo_rotated(ref, nt, U)).max() <= TOL
    po = np.arange(nt) ^ 1 if nt % 2 == 0 else np.arange(nt)
    J, K, Lm = m.jkl(po)
    Jo, Ko, Lo = o.jkl_matrices(ref, nt, po)
    assert np.abs(J - Jo).max() <= TOL and np.abs(K - Ko).max() <= TOL and np.abs(Lm - Lo).max() <= TOL


def test_hx_fock_golden():
    g = golden("hx_fock")
    n = g["hc"].shape[0]
    mc = mo.RiMoEri.from_tensor(g["Bc"], n)
    Fc = mo.hartreeExchangeFockMatrix(g["hc"], mc, g["occ"], g["h2"], g["x2"], g["po"], g["l1"], g["l2"])
    assert np.abs(Fc - g["Fc"]).max() <= TOL
    assert np.abs(mo.jkOnlyFockMatrix(g["hc"], mc, g["occ"], g["h2"], g["x2"]) - g["Fc0"]).max() <= TOL
    nsp = int(round(g["Bmo"].shape[1] ** 0.5))
    mr = mo.RiNonRelSpinMoEri.from_tensor(g["Bmo"], nsp)
    Fr = mo.hartreeExchangeFockMatrix(g["hr"], mr, g["occr"], g["h2r"], g["x2r"], g["por"], g["l1r"], g["l2r"])
    assert np.abs(Fr - g["Fr"]).max() <= TOL


@pytest.mark.parametrize("n,naux", [(16, 40), (48, 150)])
def test_hx_fock_vs_oracle(n, naux):
    rng = np.random.default_rng(n + naux)
    B = (rng.standard_normal((naux, n * n)) + 1j * rng.standard_normal((naux, n * n))) * 0.1
    h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    occ = rng.random(n)
    h2, x2, l1, l2 = (rng.standard_normal((n, n)) for _ in range(4))
    po = np.arange(n) ^ 1
    m = mo.RiMoEri.from_tensor(B, n)
    F = mo.hartreeExchangeFockMatrix(h, m, occ, h2, x2, po, l1, l2)
    Fo = o.hx_fock(h, B, occ, h2, x2, po, l1, l2)
    assert np.abs(F - Fo).max() <= TOL


def test_errors_like_reference():
    g = golden("hx_fock")
    n = g["hc"].shape[0]
    mc = mo.RiMoEri.from_tensor(g["Bc"], n)
    with pytest.raises(RrError, match="inconsistent with h"):
        mo.hartreeExchangeFockMatrix(g["hc"][:-1, :-1], mc, g["occ"], g["h2"], g["x2"])
    with pytest.raises(RrError, match="pair_of/two_rdm_l1/two_rdm_l2"):
        mo.hartreeExchangeFockMatrix(g["hc"], mc, g["occ"], g["h2"], g["x2"], g["po"], g["l1"], None)
