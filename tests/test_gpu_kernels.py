"""Unit tests of the kernel families on the GPU: the FP64 DMMA GEMM (every layout, complex,
split-K, mirror) and the TMA J streaming passes, against numpy fp64."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    return t.cpu().numpy()


def _op(a, transposed, conj):
    r = a.T if transposed else a
    return np.conj(r) if conj else r


def _run(M, N, K, opA, opB, batch=1, cplx=False, conjA=False, conjB=False, alpha=1.3, beta=0.0, mirror=0,
         split=True, seed=0):
    rng = np.random.default_rng(seed)
    dt = np.complex128 if cplx else np.float64

    def rnd(*s):
        x = rng.standard_normal(s)
        return (x + 1j * rng.standard_normal(s)) if cplx else x

    a_shape = (K, M) if opA else (M, K)
    b_shape = (N, K) if opB else (K, N)
    A = rnd(batch, *a_shape).astype(dt)
    B = rnd(batch, *b_shape).astype(dt)
    C0 = rnd(batch, M, N).astype(dt)
    ref = np.stack([alpha * _op(A[i], opA, conjA) @ _op(B[i], opB, conjB) + beta * C0[i] for i in range(batch)])
    if mirror:
        for i in range(batch):
            up = np.triu(ref[i])
            low = (up.conj().T if mirror > 0 else -up.conj().T) if cplx else (up.T if mirror > 0 else -up.T)
            ref[i] = up + np.tril(low, -1)
    dA, dB, dC = _dev(A.view(np.float64)), _dev(B.view(np.float64)), _dev(C0.view(np.float64))
    lda = a_shape[1]
    ldb = b_shape[1]
    L.check(L.lib().rr_test_gemm_f64(M, N, K, dA.data_ptr(), lda, a_shape[0] * a_shape[1], int(opA), dB.data_ptr(), ldb,
                                     b_shape[0] * b_shape[1], int(opB), dC.data_ptr(), N, M * N, alpha, beta, batch,
                                     int(cplx), int(conjA), int(conjB), mirror, int(split)))
    out = _np(dC).view(dt).reshape(batch, M, N)
    return out, ref


@pytest.mark.parametrize("opA", [0, 1])
@pytest.mark.parametrize("opB", [0, 1])
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 13, 5), (40, 400, 400), (64, 64, 64), (65, 33, 129), (3, 250, 17),
                                   (100, 100, 3000)])
def test_gemm_real_layouts(opA, opB, shape):
    M, N, K = shape
    out, ref = _run(M, N, K, opA, opB, beta=0.7)
    assert np.abs(out - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * np.sqrt(K)


@pytest.mark.parametrize("opA,opB,conjA,conjB", [(0, 0, 0, 0), (1, 0, 1, 0), (0, 1, 0, 1), (1, 1, 1, 1), (0, 1, 1, 0)])
@pytest.mark.parametrize("shape", [(5, 9, 7), (33, 70, 65), (80, 80, 200)])
def test_gemm_complex(opA, opB, conjA, conjB, shape):
    M, N, K = shape
    out, ref = _run(M, N, K, opA, opB, cplx=True, conjA=bool(conjA), conjB=bool(conjB), beta=0.5)
    assert np.abs(out - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * np.sqrt(K)


@pytest.mark.parametrize("batch", [1, 3, 37])
def test_gemm_batched_small_m(batch):
    for M in (1, 8, 13, 40, 47):
        out, ref = _run(M, 96, 80, 0, 0, batch=batch, seed=M)
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max() * 10


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("mirror", [1, -1])
def test_gemm_mirror_split(cplx, mirror):
    # A^T A style product, symmetric part kept by the mirror
    out, ref = _run(130, 130, 5000, 1, 0, cplx=cplx, mirror=mirror, split=True)
    assert np.abs(out - ref).max() <= 1e-11 * np.abs(ref).max()


def test_gemm_split_is_deterministic():
    a, _ = _run(96, 96, 20000, 1, 0, split=True, seed=5)
    b, _ = _run(96, 96, 20000, 1, 0, split=True, seed=5)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("naux,n2", [(1, 1), (3, 49), (37, 169), (129, 576), (200, 4099), (64, 20000)])
def test_j_passes(naux, n2):
    rng = np.random.default_rng(naux + n2)
    B = rng.standard_normal((naux, n2))
    D = rng.standard_normal(n2)
    dB, dD = _dev(B), _dev(D)
    g = torch.empty(naux, dtype=torch.float64, device="cuda")
    J = torch.empty(n2, dtype=torch.float64, device="cuda")
    L.check(L.lib().rr_test_j_passes(dB.data_ptr(), naux, n2, dD.data_ptr(), g.data_ptr(), J.data_ptr()))
    gref = B @ D
    Jref = B.T @ gref
    assert np.abs(_np(g) - gref).max() <= 1e-12 * np.sqrt(n2) * np.abs(gref).max()
    assert np.abs(_np(J) - Jref).max() <= 1e-12 * np.sqrt(naux * n2) * np.abs(Jref).max()


@pytest.mark.parametrize("naux,n,kind", [(1, 1, "sym"), (5, 2, "sym"), (37, 33, "sym"), (129, 64, "roundoff"),
                                         (200, 97, "roundoff"), (64, 150, "sym"), (40, 31, "asym")])
def test_j_passes_packed(naux, n, kind):
    """Packed upper-triangle passes: exact-symmetric and roundoff-symmetric B take them and match the
    dense formula; a B that is not symmetric falls back to the dense passes."""
    rng = np.random.default_rng(naux + n)
    g = rng.uniform(0.5, 1.5, size=(naux, n))
    c = rng.standard_normal((naux, n, n))
    c = c + c.transpose(0, 2, 1)
    if kind == "sym":
        B = c
    elif kind == "roundoff":  # (c g_q) g_a against (c g_a) g_q: symmetric to an ulp or two
        B = c * g[:, :, None] * g[:, None, :]
    else:
        B = c + 1e-6 * rng.standard_normal((naux, n, n))
    B = np.ascontiguousarray(B.reshape(naux, n * n))
    D = rng.standard_normal((n, n))
    dB, dD = _dev(B), _dev(D.reshape(-1))
    gam = torch.empty(naux, dtype=torch.float64, device="cuda")
    J = torch.empty(n * n, dtype=torch.float64, device="cuda")
    packed = ctypes.c_int32(-1)
    L.check(L.lib().rr_test_j_passes_packed(dB.data_ptr(), naux, n, dD.data_ptr(), gam.data_ptr(), J.data_ptr(),
                                            ctypes.byref(packed)))
    assert packed.value == (0 if kind == "asym" else 1)
    gref = B @ D.reshape(-1)
    Jref = B.T @ gref
    n2 = n * n
    assert np.abs(_np(gam) - gref).max() <= 1e-12 * np.sqrt(n2) * np.abs(gref).max()
    Jg = _np(J)
    assert np.abs(Jg - Jref).max() <= 1e-12 * np.sqrt(naux * n2) * np.abs(Jref).max()
    if kind != "asym":
        Jm = Jg.reshape(n, n)
        assert np.array_equal(Jm, Jm.T)


@pytest.mark.parametrize("nocc,n,naux", [(40, 400, 30), (17, 64, 7), (45, 82, 3), (1, 2, 1)])
def test_half_transform_variants(nocc, n, naux):
    """T[P] = Ct B^P through the general DMMA GEMM (m8n8k4) and every tiling of the m16n8k8 half-transform
    (the CTA-synchronous ring in its warp / depth / stage variants and the warp-specialised bulk-copy
    pipeline), ragged tiles included (n not a multiple of 80 or 16, nocc not a multiple of 40 or 8),
    against numpy."""
    rng = np.random.default_rng(n + nocc)
    Ct = rng.standard_normal((nocc, n))
    B = rng.standard_normal((naux, n * n))
    ref = np.einsum("ik,Pkj->Pij", Ct, B.reshape(naux, n, n), optimize=True)
    dC, dB = torch.from_numpy(Ct).cuda(), torch.from_numpy(B).cuda()
    for variant in range(15):
        T = torch.full((naux, nocc, n), float("nan"), dtype=torch.float64, device="cuda")
        L.check(L.lib().rr_test_half_transform(dC.data_ptr(), nocc, dB.data_ptr(), naux, n, T.data_ptr(), variant))
        err = np.abs(T.cpu().numpy() - ref).max()
        assert err <= 1e-12 * max(1.0, np.abs(ref).max()) * np.sqrt(n), (variant, err)
