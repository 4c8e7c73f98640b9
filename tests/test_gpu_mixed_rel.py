"""Split-BF16 relativistic exchange and the incremental (density-change) build against FP64.

* Full mixed X2C / RKB Fock matrices: within 1e-4 of max|G| of the FP64 build (as the nonrelativistic
  mixed exchange).
* Incremental builds: the change of the Fock matrix between two nearby densities is reproduced to
  1e-4 of its own size, which a difference of two full mixed builds (error ~1e-6 of |G|) cannot do
  for a change of 1e-3.
* Mixed SCF loops (X2C-HF, 4c-DHF) reach the FP64 loop's converged energy within 1e-8 Ha with a single
  FP64 build at the end."""
import numpy as np
import pytest
from scipy.linalg import expm

from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import ri, scf  # noqa: E402

REL = 1e-4


def _x2c_src(s):
    return ri.RiX2cEriSource(int(s["h"].shape[0]) // 2, s["B"], s["X"], s["S"])


def _rkb_src(s):
    return ri.RiDirectEriSource(int(s["nl"]), int(s["ns"]), s["B_LL"], s["B_SS"], s["v_total"], s["s_full"],
                                s["x_full"])


def _g_err(Fm, F64, h):
    return np.abs(Fm - F64).max() / np.abs(F64 - h).max()


@pytest.mark.parametrize("nl,naux,ne,seed", [(12, 60, 6, 21), (40, 160, 10, 22), (80, 100, 70, 5)])
def test_x2c_mixed_fock_vs_fp64(nl, naux, ne, seed):
    s = synth.x2c_system(nl, naux, ne, seed=seed)
    src = _x2c_src(s)
    F64 = ri.x2cFockMatrix(s["h"], src, s["P0"])
    Fm = ri.x2cFockMatrix(s["h"], src, s["P0"], precision="mixed")
    assert _g_err(Fm, F64, s["h"]) <= REL
    G = Fm - s["h"]  # the mixed two-electron matrix is Hermitian (mirrored blocks, real diagonal)
    assert np.abs(G - G.conj().T).max() <= 1e-13 * np.abs(Fm).max()


@pytest.mark.parametrize("nl,ns,naux,ne,seed", [(6, 11, 40, 4, 23), (12, 25, 80, 8, 24)])
def test_rkb_mixed_fock_vs_fp64(nl, ns, naux, ne, seed):
    s = synth.rkb_system(nl, ns, naux, ne, seed=seed)
    src = _rkb_src(s)
    F64 = ri.rkbFockMatrix(s["h"], src, s["P0"])
    Fm = ri.rkbFockMatrix(s["h"], src, s["P0"], precision="mixed")
    assert _g_err(Fm, F64, s["h"]) <= REL


def _rotated_density(X, S, P, ne, eps, rng):
    """Density of the occupied space of P turned by exp(eps (A - A^dagger)) in the orthonormal basis."""
    Pe = X.conj().T @ S @ P @ S @ X
    w, y = np.linalg.eigh(0.5 * (Pe + Pe.conj().T))
    Y = y[:, -ne:]
    m = Pe.shape[0]
    A = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    Y2 = expm(eps * (A - A.conj().T)) @ Y
    return X @ Y2 @ Y2.conj().T @ X.conj().T


@pytest.mark.parametrize("kind", ["x2c", "rkb"])
def test_incremental_build_tracks_the_density_change(kind):
    rng = np.random.default_rng(7)
    if kind == "x2c":
        s = synth.x2c_system(40, 160, 10, seed=22)
        src, X, S, ne = _x2c_src(s), s["X"], s["S"], 10
        build = ri.x2cFockMatrix
    else:
        s = synth.rkb_system(12, 25, 80, 8, seed=24)
        src, X, S, ne = _rkb_src(s), s["x_full"], s["s_full"], 8
        build = ri.rkbFockMatrix
    P1 = s["P0"]
    P2 = _rotated_density(X, S, P1, ne, 1e-3, rng)
    dF64 = build(s["h"], src, P2) - build(s["h"], src, P1)
    F1 = build(s["h"], src, P1, precision="mixed")                      # full build, seeds the accumulator
    F2 = build(s["h"], src, P2, precision="mixed", incremental=True)    # adds the exchange of the change
    err = np.abs((F2 - F1) - dF64).max() / np.abs(dF64).max()
    assert err <= REL, f"incremental change error {err:.2e}"
    # the same change from two full mixed builds is far less accurate
    F2f = build(s["h"], src, P2, precision="mixed")
    err_full = np.abs((F2f - F1) - dF64).max() / np.abs(dF64).max()
    assert err < 0.2 * err_full


def test_nonrel_incremental_exchange_matches_difference():
    n, naux, nocc = 160, 64, 150  # 150 occupied rows: two slices of the incremental half-transform
    rng = np.random.default_rng(9)
    B = synth.ri_tensor(n, naux, 4, box=8.0)
    C0 = np.linalg.qr(rng.standard_normal((n, nocc)))[0].T.copy()
    C1 = C0 + 1e-3 * rng.standard_normal(C0.shape)
    Bn = B.reshape(naux, n, n)

    def kref(Ct):
        T = np.einsum("iq,Pqa->Pia", Ct, Bn, optimize=True)
        return np.einsum("Pia,Pib->ab", T, T, optimize=True)

    dref = kref(C1) - kref(C0)
    dB = torch.from_numpy(B).cuda()
    d1, d0 = torch.from_numpy(C1).cuda(), torch.from_numpy(C0).cuda()
    dK = torch.empty((n, n), dtype=torch.float64, device="cuda")
    L.check(L.lib().rr_test_mixed_exchange_delta(dB.data_ptr(), naux, n, d1.data_ptr(), d0.data_ptr(), nocc,
                                                 dK.data_ptr()))
    dk = dK.cpu().numpy()
    assert np.abs(dk - dref).max() <= REL * np.abs(dref).max()
    assert np.abs(dk - dk.T).max() == 0.0


@pytest.mark.parametrize("kind", ["x2c", "dhf"])
def test_mixed_scf_reaches_fp64_energy(ref_lib, kind):
    if kind == "x2c":
        s = synth.x2c_system(40, 160, 10, seed=22)

        def run(**kw):
            return scf.runX2CHartreeFockScf(s["h"], _x2c_src(s), s["X"], s["P0"], int(s["n_electrons"]), **kw)
    else:
        s = synth.rkb_system(12, 25, 80, 8, seed=24)

        def run(**kw):
            return scf.runDiracHartreeFockScf(s["h"], _rkb_src(s), s["x_full"], s["P0"], int(s["n_electrons"]), **kw)
    r64 = run()
    rm = run(precision="mixed")
    # the reference's own FP64 loop (compiled from its sources) is the judge of the mixed energy
    rr = ref_lib.x2c_scf(s) if kind == "x2c" else ref_lib.dhf_scf(s)
    assert rr["converged"]
    assert abs(rm["energy"] - rr["energy"]) <= 1e-8
    assert r64["converged"] and rm["converged"]
    assert rm["mixed_iterations"] >= 2 and rm["fp64_iterations"] == 1
    assert rm["iterations"] == rm["mixed_iterations"] + 1
    assert abs(rm["energy"] - r64["energy"]) <= 1e-8
    assert abs(rm["history"][-1] - rm["energy"]) == 0.0
    rs = run(precision="mixed", mixed_switch=1e-4)  # one FP64 re-seed of the accumulated exchange
    assert rs["converged"] and rs["fp64_iterations"] in (1, 2)  # the re-seed happens only if |dE| gets below 1e-4 first
    assert abs(rs["energy"] - r64["energy"]) <= 1e-8
    assert abs(rs["energy"] - rr["energy"]) <= 1e-8
