"""rr_ri_coulomb_noalloc (Coulomb matrix with all scratch in a fixed device array) against the
allocating J streaming passes (rr_test_j_passes) and numpy, on two calls in a row.

Named to be collected last, so that it also runs after every other GPU test in one process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import synth  # noqa: E402
from rerdmft_b200.ri import RiStore  # noqa: E402

RTOL = 1e-12  # relative to max |J|: both paths sum FP64 in fixed orders that differ only in range splits


def _case(n, naux, seed):
    rng = np.random.default_rng(seed)
    B = synth.ri_tensor(n, naux, seed, box=8.0)
    a = rng.standard_normal((n, n))
    D = 0.5 * (a + a.T)
    return B, D


def _existing_j(B, D):
    """J through the allocating J passes (fresh scratch from cudaMalloc on every call)."""
    naux, n2 = B.shape
    dB = torch.from_numpy(B).cuda()
    dD = torch.from_numpy(D.reshape(-1)).cuda()
    gamma = torch.empty(max(naux, 1), dtype=torch.float64, device="cuda")
    J = torch.empty(n2, dtype=torch.float64, device="cuda")
    L.check(L.lib().rr_test_j_passes(dB.data_ptr(), naux, n2, dD.data_ptr(), gamma.data_ptr(), J.data_ptr()))
    return J.cpu().numpy().reshape(D.shape)


def _noalloc_dev(store, dD, dJ):
    o = L.opts(L.RR_MEM_DEVICE, sync=1)
    L.check(L.lib().rr_ri_coulomb_noalloc(store.handle, dD.data_ptr(), dJ.data_ptr(), ctypes.byref(o)))


@pytest.mark.parametrize("n,naux", [(24, 129), (33, 200), (7, 1), (400, 1600)])
def test_noalloc_matches_allocating_passes_twice(n, naux):
    B, D = _case(n, naux, seed=n + naux)
    ref = _existing_j(B, D)
    scale = max(np.abs(ref).max(), 1e-300)
    store = RiStore(B, nl=n)
    dD = torch.from_numpy(D).cuda()
    outs = []
    for _ in range(2):
        dJ = torch.full((n, n), np.nan, dtype=torch.float64, device="cuda")
        _noalloc_dev(store, dD, dJ)
        outs.append(dJ.cpu().numpy())
    for J in outs:
        assert np.abs(J - ref).max() <= RTOL * scale
    assert np.array_equal(outs[0], outs[1])
    if n <= 64:
        exact = (B.T @ (B @ D.reshape(-1))).reshape(n, n)
        assert np.abs(outs[0] - exact).max() <= 1e-11 * max(np.abs(exact).max(), 1e-300)
    store.close()


def test_noalloc_host_pointers_twice():
    n, naux = 33, 150
    B, D = _case(n, naux, seed=5)
    ref = _existing_j(B, D)
    store = RiStore(B, nl=n)
    o = L.opts(L.RR_MEM_HOST)
    outs = []
    for _ in range(2):
        J = np.full((n, n), np.nan)
        L.check(L.lib().rr_ri_coulomb_noalloc(store.handle, D.ctypes.data, J.ctypes.data, ctypes.byref(o)))
        outs.append(J)
    for J in outs:
        assert np.abs(J - ref).max() <= RTOL * np.abs(ref).max()
    assert np.array_equal(outs[0], outs[1])
    store.close()


def test_noalloc_leaves_free_memory_unchanged():
    n, naux = 200, 800
    B, D = _case(n, naux, seed=9)
    store = RiStore(B, nl=n)
    dD = torch.from_numpy(D).cuda()
    dJ = torch.empty((n, n), dtype=torch.float64, device="cuda")
    _noalloc_dev(store, dD, dJ)  # first call on the device: address lookup
    torch.cuda.synchronize()
    allocs0 = L.lib().rr_test_device_allocations()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        _noalloc_dev(store, dD, dJ)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # the library's own count of its cudaMalloc calls is the primary check; free device memory (a
    # device-wide reading that other activity could move) is the secondary one
    assert L.lib().rr_test_device_allocations() == allocs0
    assert free1 == free0
    store.close()


def test_noalloc_rejects_sizes_beyond_scratch():
    n, naux = 1500, 1  # 2 * n^2 doubles > 4,194,304
    B = np.zeros((naux, n * n))
    store = RiStore(B, nl=n)
    dD = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    dJ = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    o = L.opts(L.RR_MEM_DEVICE, sync=1)
    rc = L.lib().rr_ri_coulomb_noalloc(store.handle, dD.data_ptr(), dJ.data_ptr(), ctypes.byref(o))
    assert rc == L.RR_ERR_ARG
    assert b"needs at least" in L.lib().rr_last_error()
    store.close()
