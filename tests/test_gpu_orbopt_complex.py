"""The complex-spinor ADAM rotation problem (RotationProblem<std::complex<double>, RiMoEri>,
src/Full_opt/FullOptimization.cpp:1330-1548) on the GPU against the reference's own generalized Fock
(riHxFockGemm), orbitalGradient, spinorRotationMatrix, Adam<complex>::step and
hartreeExchangeJointHessianDiagonal (compiled oracle), and against the numpy restatement of the
RotationProblem / AdamOptimizer pair run for run."""
import numpy as np
import pytest

from oracle import ri_oracle as o
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import mo, orbopt  # noqa: E402


def _problem(f, **kw):
    eri = mo.RiMoEri.from_tensor(f["Bmo"], f["n"])
    extra = {k: f[k] for k in ("pair_of", "two_rdm_l1", "two_rdm_l2") if k in f}
    prob = orbopt.RotationProblem(eri, f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"],
                                  n_negative=f.get("n_negative", 0), **extra, **kw)
    return prob, eri


def _numpy(f):
    return o.RotationProblemComplexNumpy(f["Bmo"], f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"],
                                         f.get("pair_of"), f.get("two_rdm_l1"), f.get("two_rdm_l2"),
                                         n_negative=f.get("n_negative", 0))


@pytest.mark.parametrize("n", [6, 17, 40])
def test_complex_rotation_matrix_matches_reference(ref_lib, n):
    rng = np.random.default_rng(n)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * (0.02 * n)
    k = np.ascontiguousarray(a - a.conj().T)
    U = np.empty_like(k)
    L.check(L.lib().rr_test_rotation_matrix_complex(n, k.ctypes.data, U.ctypes.data))
    assert np.abs(U - ref_lib.rotation_matrix(k)).max() <= 1e-13
    assert np.abs(U.conj().T @ U - np.eye(n)).max() <= 1e-13


@pytest.mark.parametrize("with_pairs,n_negative", [(False, 0), (True, 0), (True, 4)])
def test_energy_gradient_joint_diagonal_vs_reference(ref_lib, with_pairs, n_negative):
    n, naux = 12, 40
    f = synth.functional_system_complex(n, naux, 3, with_pairs=with_pairs, n_negative=n_negative)
    prob, eri = _problem(f)
    args = (f.get("pair_of"), f.get("two_rdm_l1"), f.get("two_rdm_l2"))
    F = ref_lib.hx_fock_complex(f["Bmo"], n, f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"], *args)
    e_ref = 0.5 * float(np.sum(f["occupations"] * np.real(np.diag(f["h"]))) + np.real(np.trace(F)))
    assert abs(prob.energy() - e_ref) <= 1e-11 * max(1.0, abs(e_ref))
    G = ref_lib.orbital_gradient(F)
    p, q = prob.pairs[:, 0], prob.pairs[:, 1]
    assert prob.n_pairs == len(p) == (n - n_negative) * (n - n_negative - 1) // 2
    assert (q >= n_negative).all()
    g = prob.gradient()
    assert np.abs(g - G[p, q]).max() <= 1e-11 * max(1.0, np.abs(G).max())
    hd = prob.hessian_diagonal()
    hd_ref = ref_lib.hx_joint_hessian_diag(f["Bmo"], n, f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"], F,
                                           prob.pairs, *args)
    assert hd.shape == (2 * prob.n_pairs,)
    assert np.abs(hd - hd_ref).max() <= 1e-10 * max(1.0, np.abs(hd_ref).max())
    # preconditioner inputs: real parts of F, J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i)
    b3 = f["Bmo"].reshape(naux, n, n)
    d = np.einsum("Pii->Pi", b3)
    J = np.real(d.T @ d)
    K = np.real(np.einsum("Pij,Pji->ij", b3, b3))
    exp = np.stack([np.real(np.diag(F))[q], np.real(np.diag(F))[p], f["occupations"][q], f["occupations"][p],
                    J[q, p], K[q, p], J[q, q], J[p, p]], axis=1)
    assert np.abs(prob.features() - exp).max() <= 1e-5 * max(1.0, np.abs(exp).max())
    prob.close()
    eri.close()


@pytest.mark.parametrize("with_pairs,n_negative", [(False, 0), (True, 4)])
def test_adam_runs_follow_the_numpy_restatement(with_pairs, n_negative):
    n, naux = 12, 40
    f = synth.functional_system_complex(n, naux, 4, with_pairs=with_pairs, n_negative=n_negative)
    prob, eri = _problem(f)
    npb = _numpy(f)
    opt = o.AdamOptimizerNumpy()
    for _ in range(5):
        r = prob.run()
        rn = opt.run(npb)
        assert r["iterations"] == rn["iterations"]
        assert r["restart_requested"] == int(rn["restart_requested"])
        assert abs(r["energy_best"] - rn["energy_best"]) <= 1e-10
    u, hr, b = prob.state(with_tensor=True)
    assert np.abs(u.conj().T @ u - np.eye(n)).max() <= 1e-12
    assert np.abs(hr - u.conj().T @ f["h"] @ u).max() <= 1e-10
    assert np.abs(hr - npb.h).max() <= 1e-9
    assert np.abs(u - npb.u).max() <= 1e-9
    assert np.abs(b - npb.B).max() <= 1e-9
    if n_negative:
        # no pair touches the negative branch: its rows and columns of the rotation stay the identity
        assert np.abs(u[:n_negative, :n_negative] - np.eye(n_negative)).max() <= 1e-14
        assert np.abs(u[:n_negative, n_negative:]).max() <= 1e-14
        assert np.abs(u[n_negative:, :n_negative]).max() <= 1e-14
    prob.close()
    eri.close()


def test_complex_full_optimization_converges_with_and_without_scales():
    res = {}
    for mode in ("plain", "exact"):
        f = synth.functional_system_complex(10, 36, 5, nocc=3)
        prob, eri = orbopt.problem_from_system(f)
        res[mode] = orbopt.run_full_optimization(prob, exact_hessian=(mode == "exact"))
        g = prob.gradient()
        prob.close()
        eri.close()
        assert res[mode]["converged"]
        assert np.abs(g).max() < 1e-3
    assert abs(res["plain"]["energy"] - res["exact"]["energy"]) <= 1e-7
