"""The one-time set-up path on the device against the reference (a5 and the orthogonalisations of a13):

* canonicalOrthogonalize / canonicalOrthogonalizeHermitian (src/Linear_Algebra/LinearAlgebra.cpp:267-349)
  with the RankReductionReport; X is compared through X X^dagger (LAPACK and the device solver may pick
  different signs, phases or bases inside a degenerate eigenvalue) except where the reference returns the
  unique symmetric S^-1/2 (real S, nothing dropped), which is compared directly;
* the metric contraction of riThreeCenterTensor (src/AO_ints/ThreeCenterIntegrals.cpp:219-236);
* transformRiThreeCenterAoLegs (:191-217), against the fixture and the live compiled reference;
* a resident store built from raw integrals (rr_ri_create_raw) against the store built from the finished B.

Bar: max-abs 1e-10."""
import numpy as np
import pytest

from conftest import golden
from oracle import ri_oracle as o
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import ri  # noqa: E402
from rerdmft_b200._lib import RrError  # noqa: E402

TOL = 1e-10


def _rep(a):
    return [int(a[0]), int(a[1]), float(a[2]), float(a[3])]


def test_canonical_orthogonalize_golden():
    g = golden("ri_setup")
    X, rep = ri.canonicalOrthogonalize(g["metric"], 1e-10, report=True)
    assert X.shape == g["metric_x"].shape
    r = _rep(g["metric_report"])
    assert [rep["n_kept"], rep["n_dropped"]] == r[:2]
    assert abs(rep["smallest_kept"] - r[2]) <= 1e-12 and abs(rep["largest_dropped"] - r[3]) <= 1e-12
    assert np.abs(X.T @ g["metric"] @ X - np.eye(X.shape[1])).max() <= 1e-9
    assert np.abs(X @ X.T - g["metric_x"] @ g["metric_x"].T).max() <= 1e-8  # cond ~ 1e2 of the kept part
    Xf = ri.canonicalOrthogonalize(g["S_full_rank"], 1e-10)
    assert np.abs(Xf - g["X_full_rank"]).max() <= TOL
    Xh, reph = ri.canonicalOrthogonalizeHermitian(g["s_full"], 1e-10, report=True)
    assert [reph["n_kept"], reph["n_dropped"]] == _rep(g["s_full_report"])[:2]
    assert np.abs(Xh @ Xh.conj().T - g["XXh"]).max() <= TOL
    assert np.abs(Xh.conj().T @ g["s_full"] @ Xh - np.eye(Xh.shape[1])).max() <= 1e-10


def test_canonical_orthogonalize_vs_reference(ref_lib):
    k = synth.rkb_system(40, 90, 100, 8, seed=41)
    Xh, rep = ri.canonicalOrthogonalizeHermitian(k["s_full"], 1e-10, report=True)
    Xr, repr_ = ref_lib.canonical_orth_report(k["s_full"], 1e-10)
    assert Xh.shape == Xr.shape and rep["n_dropped"] == repr_["n_dropped"]
    assert abs(rep["smallest_kept"] - repr_["smallest_kept"]) <= 1e-12
    assert np.abs(Xh @ Xh.conj().T - Xr @ Xr.conj().T).max() <= TOL
    # device pointers
    dS = torch.from_numpy(k["s_full"]).cuda()
    Xd = ri.canonicalOrthogonalizeHermitian(dS, 1e-10)
    assert Xd.is_cuda and np.abs(Xd.cpu().numpy() @ Xd.cpu().numpy().conj().T - Xr @ Xr.conj().T).max() <= TOL


def test_metric_contraction_and_ao_legs_golden():
    g = golden("ri_setup")
    B = ri.riThreeCenterTensor(g["raw"], g["metric_x"])
    assert np.abs(B - g["B"]).max() <= TOL
    n_ao = g["t"].shape[0]
    assert np.abs(ri.transformRiThreeCenterAoLegs(g["B"], n_ao, g["t"]) - g["B_legs"]).max() <= TOL
    with pytest.raises(RrError, match="t row count does not match n_ao"):
        ri.transformRiThreeCenterAoLegs(g["B"], n_ao, g["t"][:-1])
    with pytest.raises(RrError, match="metric_x row count does not match"):
        ri.riThreeCenterTensor(g["raw"][:-1], g["metric_x"])


@pytest.mark.parametrize("n_ao,n_out,naux_raw", [(33, 30, 150), (120, 100, 400)])
def test_setup_vs_reference_sizes(ref_lib, n_ao, n_out, naux_raw):
    rng = np.random.default_rng(n_ao)
    raw = synth.ri_tensor(n_ao, naux_raw, n_ao, box=8.0)
    Xm, _ = ref_lib.canonical_orth_report(
        np.exp(-0.5 * ((lambda r: ((r[:, None] - r[None]) ** 2).sum(-1))(rng.uniform(0, 8, (naux_raw, 3))))), 1e-10)
    B = ri.riThreeCenterTensor(raw, Xm)
    assert np.abs(B - o.three_center_tensor(raw, Xm)).max() <= TOL
    t = rng.standard_normal((n_ao, n_out)) * 0.3
    Bl = ri.transformRiThreeCenterAoLegs(B, n_ao, t)
    assert np.abs(Bl - ref_lib.transform_ao_legs(B, n_ao, t)).max() <= TOL


def test_store_from_raw_matches_store_from_b():
    g = golden("ri_setup")
    n_ao, n_out = g["t"].shape
    st = ri.store_from_raw(g["raw"], n_ao, g["metric_x"], g["t"])
    assert (st.n, st.naux) == (n_out, g["B_legs"].shape[0])
    s = synth.nonrel_system(n_out, g["B_legs"].shape[0], 2, seed=5)
    src = ri.RiNonRelEriSource(n_out, g["B_legs"], s["X"], s["S"])
    src_raw = ri.RiNonRelEriSource(n_out, g["B_legs"], s["X"], s["S"])
    src_raw._store = st
    F = ri.nonRelFockMatrix(s["h"], src, s["D0"])
    Fr = ri.nonRelFockMatrix(s["h"], src_raw, s["D0"])
    assert np.abs(F - Fr).max() <= TOL
    Fo = o.nonrel_fock(s["h"], g["B_legs"], s["D0"], s["S"], s["X"])
    assert np.abs(Fr - Fo).max() <= TOL
    # without t: n = n_ao, B = metric_x^T raw
    st2 = ri.store_from_raw(torch.from_numpy(g["raw"]).cuda(), n_ao, torch.from_numpy(g["metric_x"]).cuda())
    assert (st2.n, st2.naux) == (n_ao, g["B"].shape[0])
    st.close()
    st2.close()
