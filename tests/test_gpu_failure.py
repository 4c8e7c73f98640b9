"""Failure detection on the GPU without a fault: a bounded mbarrier wait that nothing completes runs out,
records its code in the status word and returns, the hook reports RR_ERR_TIMEOUT (as every TMA
pipeline of the library does; the reference's Fock builds throw std::runtime_error at their error
points, src/NON_REL/NonRelFockMatrixRi.cpp:30-36), and the context stays usable afterwards.

Nothing here faults, traps or hangs a GPU: no bulk copy is in flight while the wait runs, and the
wait itself is limited to at most 65,536 polls."""
import ctypes
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from oracle import ri_oracle  # noqa: E402
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import synth  # noqa: E402
from rerdmft_b200.ri import RiStore  # noqa: E402

EXPIRY_CODE = 0x40


def _expire(limit, threads=128):
    word, ms, cyc = ctypes.c_int32(0), ctypes.c_double(0.0), ctypes.c_double(0.0)
    t0 = time.perf_counter()
    rc = L.lib().rr_test_wait_expiry(limit, threads, ctypes.byref(word), ctypes.byref(ms), ctypes.byref(cyc))
    return rc, word.value, ms.value, cyc.value, time.perf_counter() - t0


@pytest.mark.parametrize("limit", [1 << 10, 1 << 16])
def test_bounded_wait_expires_with_timeout_status(limit):
    rc, word, ms, cycles, wall = _expire(limit)
    assert rc == L.RR_ERR_TIMEOUT, L.lib().rr_last_error()
    assert word == EXPIRY_CODE
    assert b"wait bound expired" in L.lib().rr_last_error()
    assert wall < 10.0  # the expiry is bounded: a short limit ends in well under a second
    assert cycles > 0
    print(f"wait limit {limit}: {ms:.3f} ms on the device, {cycles / limit:.1f} SM cycles per poll")


def test_context_usable_after_expired_wait():
    rc, word, *_ = _expire(1 << 12, threads=1024)
    assert rc == L.RR_ERR_TIMEOUT and word == EXPIRY_CODE
    # a normal RI Fock build on the same context afterwards
    s = synth.nonrel_system(20, 60, 4, seed=3)
    store = RiStore(s["B"], nl=20)
    F = np.empty((20, 20))
    o = L.opts(L.RR_MEM_HOST)
    L.check(L.lib().rr_ri_fock_nonrel(store.handle, s["h"].ctypes.data, s["D0"].ctypes.data, s["S"].ctypes.data,
                                      s["X"].ctypes.data, s["X"].shape[1], F.ctypes.data, ctypes.byref(o)))
    Fo = ri_oracle.nonrel_fock(s["h"], s["B"], s["D0"], s["S"], s["X"])
    assert np.abs(F - Fo).max() <= 1e-10
    store.close()


def test_wait_expiry_rejects_out_of_range_limits():
    assert _expire(0)[0] == L.RR_ERR_ARG
    assert _expire((1 << 22) + 1)[0] == L.RR_ERR_ARG
    assert _expire(16, threads=33)[0] == L.RR_ERR_ARG
