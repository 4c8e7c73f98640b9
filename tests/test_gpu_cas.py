"""The CASSCF RI operators on the device (casTwoElectronOperator, casActiveCumulantFock, casActiveIntegrals
on RiNonRelSpinMoEri and RiMoEri, src/MCSCF/CasFock.cpp:246-262) against the reference's own code compiled
from its sources.  Bar: max-abs 1e-10."""
import numpy as np
import pytest

from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import mo  # noqa: E402

TOL = 1e-10


def _tensor(n, naux, cplx, seed):
    rng = np.random.default_rng(seed)
    if cplx:
        B = 0.1 * (rng.standard_normal((naux, n * n)) + 1j * rng.standard_normal((naux, n * n)))
        return rng, B, mo.RiMoEri.from_tensor(B, n), n
    B = synth.ri_tensor(n, naux, seed, box=6.0)
    return rng, B, mo.RiNonRelSpinMoEri.from_tensor(B, n), 2 * n


def _rho(rng, d, rank, cplx):
    """A one-particle density of the given rank (the rest of the spectrum exactly zero: the low-rank
    factorisation drops it), eigenvalues in (0, 1]."""
    A = rng.standard_normal((d, d)) + (1j * rng.standard_normal((d, d)) if cplx else 0)
    q, _ = np.linalg.qr(A)
    w = np.zeros(d)
    w[:rank] = rng.uniform(0.05, 1.0, rank)
    return (q * w) @ q.conj().T


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n,naux,rank", [(6, 20, 4), (40, 150, 30)])
def test_two_electron_operator(ref_lib, cplx, n, naux, rank):
    rng, B, eri, d = _tensor(n, naux, cplx, n + naux)
    rho = _rho(rng, d, rank, cplx)
    G = mo.casTwoElectronOperator(eri, rho)
    assert np.abs(G - ref_lib.cas_two_electron(B, n, rho)).max() <= TOL
    eri.close()


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n,naux,active", [(6, 20, [0, 2, 5]), (40, 150, list(range(10, 22)))])
def test_active_cumulant_fock_and_integrals(ref_lib, cplx, n, naux, active):
    rng, B, eri, d = _tensor(n, naux, cplx, 2 * n + naux)
    a = len(active)
    lam = rng.standard_normal(a ** 4) + (1j * rng.standard_normal(a ** 4) if cplx else 0)
    F = mo.casActiveCumulantFock(eri, active, lam)
    assert np.abs(F - ref_lib.cas_cumulant_fock(B, n, active, lam)).max() <= TOL
    I = mo.casActiveIntegrals(eri, active)
    assert np.abs(I - ref_lib.cas_active_integrals(B, n, active)).max() <= TOL
    eri.close()


def test_active_index_out_of_range():
    rng, B, eri, d = _tensor(5, 12, False, 3)
    from rerdmft_b200._lib import RrError
    with pytest.raises(RrError, match="active index out of range"):
        mo.casActiveIntegrals(eri, [0, d])
    eri.close()
