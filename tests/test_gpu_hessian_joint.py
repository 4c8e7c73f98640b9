"""The complex label source of the learned preconditioner on the device: hartreeExchangeJointHessianDiagonal
on a RiMoEri (src/Hessian_opt/HartreeExchangeHessian.cpp:653-711), with and without pair terms, and with a
PNOF functional's full two-RDM (buildPnofFullTwoRdm / buildPnofPairOf, src/Hessian_opt/PnofFock.cpp), i.e.
pnofJointHessianDiagonal (src/Hessian_opt/PnofHessian.cpp:171-181), against the reference compiled from its
sources.  Bar: max-abs 1e-10."""
import numpy as np
import pytest

from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import mo  # noqa: E402
from rerdmft_b200._lib import RrError  # noqa: E402

TOL = 1e-10


def _system(n, naux, seed):
    """A Hermitian complex MO tensor B_mo^P = U^dagger B^P U (real symmetric B^P, unitary U) and a complex
    Hermitian h."""
    rng = np.random.default_rng(seed)
    B = synth.ri_tensor(n, naux, seed, box=6.0).reshape(naux, n, n)
    U = synth.random_unitary(n, rng)
    Bmo = np.einsum("ai,Pab,bj->Pij", U.conj(), B, U, optimize=True).reshape(naux, n * n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return rng, np.ascontiguousarray(Bmo), 0.5 * (A + A.conj().T)


def _gnof_geminals(n):
    """Kramers-pair geminals (2k, 2k+1), two subspaces, the first geminal of each principal."""
    g = [(2 * k, 2 * k + 1, k % 2, 1 if k < 2 else 0) for k in range(n // 2)]
    occ = np.empty(n)
    for k in range(n // 2):
        occ[2 * k] = occ[2 * k + 1] = 0.96 - 0.01 * k if k < 2 else 0.04 / (k + 1)
    return g, occ


@pytest.mark.parametrize("with_pairs", [False, True])
def test_joint_diagonal_random_rdms(ref_lib, with_pairs):
    n, naux = 16, 50
    rng, Bmo, h = _system(n, naux, 5)
    occ = rng.random(n)
    h2, x2 = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    F = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    pairs = [(p, q) for p in range(n) for q in range(p)]
    kw = {}
    if with_pairs:
        kw = dict(pair_of=np.arange(n) ^ 1, two_rdm_l1=rng.standard_normal((n, n)),
                  two_rdm_l2=rng.standard_normal((n, n)))
    eri = mo.RiMoEri.from_tensor(Bmo, n)
    d = mo.hartreeExchangeJointHessianDiagonal(h, eri, occ, h2, x2, F, pairs, **kw)
    dr = ref_lib.hx_joint_hessian_diag(Bmo, n, h, occ, h2, x2, F, pairs, kw.get("pair_of"), kw.get("two_rdm_l1"),
                                       kw.get("two_rdm_l2"))
    assert np.abs(d - dr).max() <= TOL
    eri.close()


@pytest.mark.parametrize("functional", ["PNOF5", "GNOF"])
def test_pnof_joint_diagonal(ref_lib, functional):
    """pnofJointHessianDiagonal: the PNOF full two-RDM (the reference's builder) through the device diagonal,
    with the generalized Fock matrix of the same two-RDM from the device (rr_mo_hx_fock)."""
    n, naux = 24, 80
    rng, Bmo, h = _system(n, naux, 9)
    g, occ = _gnof_geminals(n)
    full = ref_lib.pnof_full_two_rdm(functional, g, occ, n)
    eri = mo.RiMoEri.from_tensor(Bmo, n)
    F = mo.hartreeExchangeFockMatrix(h, eri, occ, full["two_rdm_h"], full["two_rdm_x"], full["pair_of"],
                                     full["two_rdm_l1"], full["two_rdm_l2"])
    pairs = [(p, q) for p in range(n) for q in range(p)]
    d = mo.hartreeExchangeJointHessianDiagonal(h, eri, occ, full["two_rdm_h"], full["two_rdm_x"], F, pairs,
                                               full["pair_of"], full["two_rdm_l1"], full["two_rdm_l2"])
    dr = ref_lib.hx_joint_hessian_diag(Bmo, n, h, occ, full["two_rdm_h"], full["two_rdm_x"], F, pairs,
                                       full["pair_of"], full["two_rdm_l1"], full["two_rdm_l2"])
    assert np.abs(d - dr).max() <= TOL
    eri.close()


def test_real_tensor_is_unsupported():
    B = synth.ri_tensor(4, 10, 1, box=4.0)
    eri = mo.RiNonRelSpinMoEri.from_tensor(B, 4)
    with pytest.raises(RrError):
        mo.hartreeExchangeJointHessianDiagonal(np.eye(8), eri, np.ones(8), np.eye(8), np.eye(8), np.eye(8), [(1, 0)])
    eri.close()
