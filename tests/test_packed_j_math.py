"""The packed-triangle form of the Coulomb passes, restated in numpy (no GPU): the row-by-row upper
triangle index, the density fold and the few-ulp symmetry test that the store applies before it
streams half of B.  gamma_P = sum_{q<=a} B^P_qa fold(D)_qa and J_qa = J_aq = sum_P gamma_P B^P_qa
must equal the reference's dense formula (gamma = B vec D, J = B^T gamma) for a symmetric B."""
import numpy as np
import pytest

EPS = np.finfo(np.float64).eps


def tri_index(q, a, n):
    return q * (2 * n - q + 1) // 2 + (a - q)


def tri_len(n):
    return n * (n + 1) // 2


def pack(B, n):
    """Upper triangles row by row, and the store's symmetry test (8 eps of the larger element)."""
    iu = np.triu_indices(n)
    b3 = B.reshape(-1, n, n)
    up, lo = b3[:, iu[0], iu[1]], b3[:, iu[1], iu[0]]
    ok = bool(np.all(np.abs(up - lo) <= 8.0 * EPS * np.maximum(np.abs(up), np.abs(lo))))
    return up, ok


def fold(D, n):
    iu = np.triu_indices(n)
    out = D[iu] + D.T[iu]
    diag = iu[0] == iu[1]
    out[diag] = D[iu][diag]
    return out


def unpack_sym(v, n):
    J = np.zeros((n, n))
    iu = np.triu_indices(n)
    J[iu] = v
    J[(iu[1], iu[0])] = v
    return J


@pytest.mark.parametrize("n", [1, 2, 3, 7, 32, 33])
def test_tri_index_is_row_major_upper_triangle(n):
    k = 0
    for q in range(n):
        for a in range(q, n):
            assert tri_index(q, a, n) == k
            k += 1
    assert k == tri_len(n)


@pytest.mark.parametrize("naux,n", [(1, 1), (5, 4), (37, 33), (64, 50)])
def test_packed_passes_equal_dense_formula(naux, n):
    rng = np.random.default_rng(naux * 100 + n)
    c = rng.standard_normal((naux, n, n))
    g = rng.uniform(0.5, 1.5, size=(naux, n))
    B = ((c + c.transpose(0, 2, 1)) * g[:, :, None] * g[:, None, :]).reshape(naux, n * n)  # roundoff-symmetric
    D = rng.standard_normal((n, n))  # the passes take any density, symmetric or not
    Bpk, ok = pack(B, n)
    assert ok
    gamma = Bpk @ fold(D, n)
    J = unpack_sym(Bpk.T @ gamma, n)
    gref = B @ D.reshape(-1)
    Jref = (B.T @ gref).reshape(n, n)
    assert np.abs(gamma - gref).max() <= 1e-12 * max(1.0, np.abs(gref).max())
    assert np.abs(J - Jref).max() <= 1e-12 * max(1.0, np.abs(Jref).max())
    assert np.array_equal(J, J.T)


def test_symmetry_test_rejects_a_real_asymmetry():
    rng = np.random.default_rng(3)
    naux, n = 4, 9
    c = rng.standard_normal((naux, n, n))
    B = (c + c.transpose(0, 2, 1)).reshape(naux, n * n)
    assert pack(B, n)[1]
    A = rng.standard_normal((naux, n, n))
    Bs = (B.reshape(naux, n, n) + 1e-12 * (A - A.transpose(0, 2, 1))).reshape(naux, n * n)
    assert not pack(Bs, n)[1]
