"""Exchange identities the CUDA builds rely on, restated in numpy (no GPU).

* Gauss's three real products for an off-diagonal relativistic exchange block
  K_fu = sum_i conj(T_f(i, a)) T_u(i, b):  with P1 = Re_f^T Re_u, P2 = Im_f^T Im_u and
  P3 = (Re_f - Im_f)^T (Re_u + Im_u),  Re K = P1 + P2 and Im K = P3 - P1 + P2.
* The incremental (density-change) build: K(C) - K(C') = X + X^dagger with
  X = sum (W B)^dagger (U B), W = (C + C') / 2, U = C - C'."""
import numpy as np
import pytest


@pytest.mark.parametrize("kk,ff,fu", [(1, 1, 1), (7, 5, 9), (64, 20, 33)])
def test_gauss_three_products(kk, ff, fu):
    rng = np.random.default_rng(kk + ff + fu)
    Tf = rng.standard_normal((kk, ff)) + 1j * rng.standard_normal((kk, ff))
    Tu = rng.standard_normal((kk, fu)) + 1j * rng.standard_normal((kk, fu))
    K = Tf.conj().T @ Tu
    rf, i_f, ru, iu = Tf.real, Tf.imag, Tu.real, Tu.imag
    p1, p2, p3 = rf.T @ ru, i_f.T @ iu, (rf - i_f).T @ (ru + iu)
    assert np.allclose(p1 + p2, K.real, rtol=0, atol=1e-12 * max(1.0, np.abs(K).max()))
    assert np.allclose(p3 - p1 + p2, K.imag, rtol=0, atol=1e-12 * max(1.0, np.abs(K).max()))


@pytest.mark.parametrize("cplx", [False, True])
def test_incremental_exchange_identity(cplx):
    rng = np.random.default_rng(5 + cplx)
    naux, r, n = 6, 4, 9
    B = rng.standard_normal((naux, n, n))
    B = B + B.transpose(0, 2, 1)

    def rows(shape):
        x = rng.standard_normal(shape)
        return x + 1j * rng.standard_normal(shape) if cplx else x

    C, C0 = rows((r, n)), rows((r, n))

    def kmat(c):
        t = np.einsum("iq,Pqa->Pia", c, B)
        return np.einsum("Pia,Pib->ab", t.conj(), t)

    W, U = 0.5 * (C + C0), C - C0
    X = np.einsum("Pia,Pib->ab", np.einsum("iq,Pqa->Pia", W, B).conj(), np.einsum("iq,Pqa->Pia", U, B))
    d = kmat(C) - kmat(C0)
    assert np.abs((X + X.conj().T) - d).max() <= 1e-12 * max(1.0, np.abs(d).max())
