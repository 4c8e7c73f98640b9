"""The split-BF16 tcgen05 exchange (RR_PREC_MIXED) against FP64.

Three BF16 products per FP64 product with FP32 accumulation give ~2^-16 relative error per
element; the bound used here, 1e-4 of max|K|, leaves room for the accumulation over n*nocc*naux."""
import ctypes

import numpy as np
import pytest

from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import ri  # noqa: E402

REL = 1e-4


def _mixed_k(B, Ct):
    naux, n2 = B.shape
    n = int(round(n2 ** 0.5))
    dB = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(Ct)).cuda()
    K = torch.empty((n, n), dtype=torch.float64, device="cuda")
    L.check(L.lib().rr_test_mixed_exchange(dB.data_ptr(), naux, n, dC.data_ptr(), Ct.shape[0], K.data_ptr()))
    return K.cpu().numpy()


def _ref_k(B, Ct):
    naux = B.shape[0]
    n = Ct.shape[1]
    T = np.einsum("iq,Pqa->Pia", Ct, B.reshape(naux, n, n), optimize=True)
    return np.einsum("Pia,Pib->ab", T, T, optimize=True)


@pytest.mark.parametrize("naux,n,nocc", [(1, 8, 1), (8, 64, 8), (37, 100, 40), (20, 130, 50), (64, 129, 7),
                                         (200, 400, 40)])
def test_mixed_exchange_accuracy(naux, n, nocc):
    rng = np.random.default_rng(naux * 1000 + n)
    B = synth.ri_tensor(n, naux, naux + n, box=8.0)
    Ct = np.linalg.qr(rng.standard_normal((n, nocc)))[0].T.copy()
    K = _mixed_k(B, Ct)
    Kr = _ref_k(B, Ct)
    err = np.abs(K - Kr).max() / max(np.abs(Kr).max(), 1e-300)
    assert err <= REL, f"relative error {err:.2e}"
    assert np.abs(K - K.T).max() == 0.0  # mirrored exactly


def test_mixed_is_deterministic():
    rng = np.random.default_rng(3)
    B = synth.ri_tensor(96, 64, 3, box=8.0)
    Ct = rng.standard_normal((24, 96))
    a = _mixed_k(B, Ct)
    b = _mixed_k(B, Ct)
    assert np.array_equal(a, b)


def test_jk_occupied_mixed_vs_fp64():
    n, naux, nocc = 200, 300, 20
    s = synth.nonrel_system(n, naux, nocc, seed=11)
    rng = np.random.default_rng(12)
    C, _ = synth.occupied_density(n, nocc, rng)
    store = ri.RiStore(s["B"], nl=n)
    J64, K64 = ri.jk_occupied(store, C)
    Cd = torch.from_numpy(C).cuda()
    Jm = torch.empty((n, n), dtype=torch.float64, device="cuda")
    Km = torch.empty_like(Jm)
    o = L.opts(L.RR_MEM_DEVICE, precision=L.RR_PREC_MIXED)
    L.check(L.lib().rr_ri_jk_occupied(store.handle, Cd.data_ptr(), nocc, Jm.data_ptr(), Km.data_ptr(), ctypes.byref(o)))
    torch.cuda.synchronize()
    assert np.abs(Jm.cpu().numpy() - J64).max() <= 1e-12 * np.abs(J64).max()  # Coulomb stays FP64
    assert np.abs(Km.cpu().numpy() - K64).max() <= REL * np.abs(K64).max()
