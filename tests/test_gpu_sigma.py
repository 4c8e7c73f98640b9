"""The RI sigma-vector Hessian-vector primitives on the device against the reference's own
src/Hessian_opt/RiSigmaGemm.cpp and RiSigmaHessianToolkit.cpp (compiled from its sources), real and
complex, host and device pointers.  Bar: max-abs 1e-10."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402

TOL = 1e-10


def _case(n, naux, cplx, seed):
    rng = np.random.default_rng(seed)
    B = 0.1 * rng.standard_normal((naux, n * n))
    if cplx:
        B = B + 0.1j * rng.standard_normal((naux, n * n))
    K = rng.standard_normal((n, n))
    return rng, B, K - K.T


def _toolkit(B, n, K):
    cplx = np.iscomplexobj(B)
    naux = B.shape[0]
    dt = np.complex128 if cplx else np.float64
    out = dict(kb1=np.empty((naux, n * n), dt), kb2=np.empty((naux, n * n), dt), bdiag=np.empty((naux, n), dt),
               kb1diag=np.empty((naux, n), dt), kb2diag=np.empty((naux, n), dt))
    o = L.opts(L.RR_MEM_HOST)
    L.check(L.lib().rr_sigma_toolkit(B.ctypes.data, n, naux, 1 if cplx else 0, K.ctypes.data,
                                     *(out[k].ctypes.data for k in ("kb1", "kb2", "bdiag", "kb1diag", "kb2diag")),
                                     ctypes.byref(o)))
    return out


def _pair_op(op, keep):
    """rr_pair_op from an operand dict (arrays kept alive in `keep`)."""
    def p(a, dt=None):
        if a is None:
            return None
        a = np.ascontiguousarray(a) if dt is None else np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data
    s = op.get("s")
    return L.PairOp(p(s), p(op.get("idx"), np.uint32) if s is not None else None, p(op.get("w"), np.float64),
                    p(op.get("row")), p(op.get("post"), np.float64))


def _pair(target, sign, n, naux, f, g, cplx):
    keep = []
    out = np.array(target, dtype=np.complex128 if cplx else np.float64, copy=True)
    pf, pg = _pair_op(f, keep), _pair_op(g, keep)
    o = L.opts(L.RR_MEM_HOST)
    L.check(L.lib().rr_sigma_pair_contract(out.ctypes.data, sign, n, naux, 1 if cplx else 0, ctypes.byref(pf),
                                           ctypes.byref(pg), ctypes.byref(o)))
    return out


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n,naux", [(6, 9), (40, 120)])
def test_toolkit(ref_lib, cplx, n, naux):
    rng, B, K = _case(n, naux, cplx, n + naux)
    got = _toolkit(B, n, K)
    want = ref_lib.sigma_toolkit(B, n, K)
    for k in want:
        assert np.abs(got[k] - want[k]).max() <= TOL, k


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n,naux", [(5, 7), (40, 120)])
def test_pair_diag_accum(ref_lib, cplx, n, naux):
    rng, B, K = _case(n, naux, cplx, 3 * n + naux)
    t = ref_lib.sigma_toolkit(B, n, K)
    T0 = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    # operands in the shapes the reference's functional code builds: tensor gathers with index tables
    # (transposed / permuted layouts), weights, per-(P,t) row factors and a post factor
    f = dict(s=B, idx=np.array([x * n + tt for tt in range(n) for x in range(n)], dtype=np.uint32),
             w=rng.standard_normal(n * n), row=t["kb1diag"], post=rng.standard_normal((n, n)))
    g = dict(s=t["kb1"], idx=rng.permutation(n * n).astype(np.uint32))
    for sign, ff, gg in ((-0.5, f, g), (1.0, dict(w=rng.standard_normal(n * n), row=t["bdiag"]), g),
                         (2.0, dict(s=t["kb2"], idx=np.arange(n * n, dtype=np.uint32)), f)):
        got = _pair(T0, sign, n, naux, ff, gg, cplx)
        want = ref_lib.sigma_pair_contract(T0, sign, n, naux, ff, gg)
        assert np.abs(got - want).max() <= TOL
    for Ua, Ub in ((t["kb1diag"], t["bdiag"]), (None, t["kb2diag"]), (t["bdiag"], None)):
        out = np.array(T0, dtype=np.complex128 if cplx else np.float64, copy=True)
        ua = None if Ua is None else np.ascontiguousarray(Ua)
        ub = None if Ub is None else np.ascontiguousarray(Ub)
        L.check(L.lib().rr_sigma_diag_contract(out.ctypes.data, n, naux, 1 if cplx else 0, B.ctypes.data,
                                               None if ua is None else ua.ctypes.data,
                                               None if ub is None else ub.ctypes.data,
                                               ctypes.byref(L.opts(L.RR_MEM_HOST))))
        assert np.abs(out - ref_lib.sigma_diag_contract(T0, n, naux, B, Ua, Ub)).max() <= TOL
    U0 = np.ascontiguousarray(t["bdiag"])
    D = np.ascontiguousarray(t["kb2diag"]).reshape(-1)
    W = rng.standard_normal((n, n))
    out = U0.copy()
    L.check(L.lib().rr_sigma_accum_u(out.ctypes.data, 0.7, n, naux, 1 if cplx else 0, D.ctypes.data, W.ctypes.data,
                                     ctypes.byref(L.opts(L.RR_MEM_HOST))))
    assert np.abs(out - ref_lib.sigma_accum_u(U0, 0.7, n, naux, D, W)).max() <= TOL


def test_device_pointers_keep_results_on_the_device(ref_lib):
    n, naux = 24, 60
    rng, B, K = _case(n, naux, True, 7)
    dB, dK = torch.from_numpy(B).cuda(), torch.from_numpy(K).cuda()
    outs = [torch.empty((naux, n * n), dtype=torch.complex128, device="cuda") for _ in range(2)]
    diags = [torch.empty((naux, n), dtype=torch.complex128, device="cuda") for _ in range(3)]
    o = L.opts(L.RR_MEM_DEVICE, sync=1)
    L.check(L.lib().rr_sigma_toolkit(dB.data_ptr(), n, naux, 1, dK.data_ptr(), *(x.data_ptr() for x in outs),
                                     *(x.data_ptr() for x in diags), ctypes.byref(o)))
    want = ref_lib.sigma_toolkit(B, n, K)
    assert np.abs(outs[0].cpu().numpy() - want["kb1"]).max() <= TOL
    assert np.abs(diags[2].cpu().numpy() - want["kb2diag"]).max() <= TOL
    T = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    idx = torch.from_numpy(np.arange(n * n, dtype=np.int32)).cuda()
    f = L.PairOp(dB.data_ptr(), idx.data_ptr(), None, None, None)
    g = L.PairOp(outs[1].data_ptr(), idx.data_ptr(), None, None, None)
    L.check(L.lib().rr_sigma_pair_contract(T.data_ptr(), 1.0, n, naux, 1, ctypes.byref(f), ctypes.byref(g),
                                           ctypes.byref(o)))
    ident = dict(idx=np.arange(n * n, dtype=np.uint32))
    ref = ref_lib.sigma_pair_contract(np.zeros((n, n), complex), 1.0, n, naux, dict(s=B, **ident),
                                      dict(s=want["kb2"], **ident))
    assert np.abs(T.cpu().numpy() - ref).max() <= TOL
