"""Functional-stage orbital optimisation on the GPU against the reference's own ADAM, rotation,
gradient, energy and Hessian code (compiled oracle) and the numpy restatement of the
RotationProblem / AdamOptimizer pair; the preconditioner MLP's training kernels against a float64
numpy restatement."""
import ctypes

import numpy as np
import pytest

from mlp_numpy import loss_and_grad as np_loss_and_grad
from oracle import ri_oracle as o
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import mo, orbopt  # noqa: E402


def _p(a):
    return a.ctypes.data


def test_adam_steps_match_reference(ref_lib):
    rng = np.random.default_rng(0)
    g = rng.standard_normal((12, 37)) * np.logspace(-3, 1, 37)
    out = np.empty_like(g)
    L.check(L.lib().rr_test_adam_steps(37, 0, 12, 0.01, 0.7, 0.9, 1e-15, _p(g), _p(out)))
    assert np.array_equal(out, ref_lib.adam_steps(g))
    gc = np.ascontiguousarray(g + 1j * rng.standard_normal(g.shape))
    outc = np.empty_like(gc)
    L.check(L.lib().rr_test_adam_steps(37, 1, 12, 0.02, 0.7, 0.9, 1e-15, _p(gc), _p(outc)))
    ref = ref_lib.adam_steps(gc, lr=0.02)
    assert np.abs(outc - ref).max() <= 1e-15 * np.abs(ref).max()


@pytest.mark.parametrize("n,scale", [(5, 0.01), (24, 0.3), (40, 3.0)])
def test_rotation_matrix_matches_reference(ref_lib, n, scale):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) * scale
    k = np.ascontiguousarray(a - a.T)
    U = np.empty_like(k)
    L.check(L.lib().rr_test_rotation_matrix(n, _p(k), _p(U)))
    assert np.abs(U - ref_lib.rotation_matrix(k)).max() <= 1e-13
    assert np.abs(U.T @ U - np.eye(n)).max() <= 1e-13


def test_adam_run_logic_matches_reference(ref_lib):
    rng = np.random.default_rng(5)
    n = 30
    a = np.logspace(-1, 3, n)
    b = rng.standard_normal(n)
    x0 = rng.standard_normal(n) * 0.1
    runs = 14
    eb, it, rs, lr, x = np.empty(runs), np.empty(runs, np.int32), np.empty(runs, np.int32), np.empty(runs), np.empty(n)
    L.check(L.lib().rr_test_adam_run_quadratic(n, _p(a), _p(b), 0.05, _p(x0), runs, _p(eb), _p(it), _p(rs), _p(lr),
                                               _p(x)))
    r = ref_lib.adam_run_quadratic(a, b, 0.05, x0, runs)
    assert np.array_equal(it, r["iterations"])
    assert np.array_equal(rs.astype(bool), r["restart"])
    assert np.array_equal(lr, r["rate"])
    assert np.abs(eb - r["energy_best"]).max() <= 1e-12 * max(1.0, np.abs(eb).max())
    assert np.abs(x - r["x"]).max() <= 1e-10


def _system(ns, naux, seed, with_pairs=False, nocc=None):
    f = synth.functional_system(ns, naux, seed, nocc=nocc, with_pairs=with_pairs)
    extra = {k: f[k] for k in ("pair_of", "two_rdm_l1", "two_rdm_l2") if k in f}
    return f["Bmo"], f["h"], f["occupations"], f["two_rdm_h"], f["two_rdm_x"], extra


def _problem(Bmo, h, occ, h2, x2, extra):
    eri = mo.RiNonRelSpinMoEri.from_tensor(Bmo, h.shape[0])
    return orbopt.RotationProblem(eri, h, occ, h2, x2, **extra), eri


@pytest.mark.parametrize("with_pairs", [False, True])
def test_energy_gradient_hessian_vs_reference(ref_lib, with_pairs):
    ns, naux = 6, 24
    Bmo, h, occ, h2, x2, extra = _system(ns, naux, 3, with_pairs)
    prob, eri = _problem(Bmo, h, occ, h2, x2, extra)
    args = (extra.get("pair_of"), extra.get("two_rdm_l1"), extra.get("two_rdm_l2"))
    H = np.zeros((2 * ns, 2 * ns))
    H[:ns, :ns] = h
    H[ns:, ns:] = h
    e_ref = ref_lib.hx_energy_nonrel(Bmo, ns, H, occ, h2, x2, *args)
    assert abs(prob.energy() - e_ref) <= 1e-11 * max(1.0, abs(e_ref))
    npb = o.RotationProblemNumpy(Bmo, h, occ, h2, x2, *args)
    assert np.abs(prob.gradient() - npb.gradient()).max() <= 1e-11
    F = ref_lib.hx_fock_nonrel(Bmo, ns, H, occ, h2, x2, *args)
    hd_ref = ref_lib.hx_hessian_diag_nonrel(Bmo, ns, H, occ, h2, x2, F, prob.pairs, *args)
    assert np.abs(prob.hessian_diagonal() - hd_ref).max() <= 1e-10 * max(1.0, np.abs(hd_ref).max())
    f = prob.features()
    J, K, _ = o.jkl_matrices(o.nonrel_mo_embedded(Bmo, ns), 2 * ns)
    p, q = prob.pairs[:, 0], prob.pairs[:, 1]
    exp = np.stack([np.diag(F)[q], np.diag(F)[p], occ[q], occ[p], J[q, p], K[q, p], J[q, q], J[p, p]], axis=1)
    assert np.abs(f - exp).max() <= 1e-5 * max(1.0, np.abs(exp).max())
    prob.close()


def test_adam_runs_follow_the_numpy_restatement():
    ns, naux = 6, 24
    Bmo, h, occ, h2, x2, extra = _system(ns, naux, 4)
    prob, eri = _problem(Bmo, h, occ, h2, x2, extra)
    npb = o.RotationProblemNumpy(Bmo, h, occ, h2, x2)
    opt = o.AdamOptimizerNumpy()
    for _ in range(4):
        r = prob.run()
        rn = opt.run(npb)
        assert r["iterations"] == rn["iterations"]
        assert r["restart_requested"] == int(rn["restart_requested"])
        assert abs(r["energy_best"] - rn["energy_best"]) <= 1e-10
    u, hr, b = prob.state(with_tensor=True)
    assert np.abs(u.T @ u - np.eye(ns)).max() <= 1e-12
    assert np.abs(hr - u.T @ h @ u).max() <= 1e-10
    assert np.abs(hr - npb.h).max() <= 1e-9
    prob.close()


def test_full_optimization_converges_and_exact_preconditioner_helps():
    ns, naux = 8, 32
    res = {}
    for mode in ("plain", "exact"):
        Bmo, h, occ, h2, x2, extra = _system(ns, naux, 3, nocc=3)
        prob, eri = _problem(Bmo, h, occ, h2, x2, extra)
        res[mode] = orbopt.run_full_optimization(prob, exact_hessian=(mode == "exact"))
        prob.close()
    assert res["plain"]["converged"] and res["exact"]["converged"]
    assert abs(res["plain"]["energy"] - res["exact"]["energy"]) <= 1e-7
    assert res["exact"]["macro_iterations"] < res["plain"]["macro_iterations"]


def test_mlp_gradient_matches_numpy():
    rng = np.random.default_rng(7)
    X = rng.standard_normal((300, 8)).astype(np.float32) * np.array([1, 2, 0.1, 0.3, 5, 1, 2, 3], np.float32)
    y = (X[:, 0] - 0.5 * X[:, 4] + np.sin(X[:, 1])).astype(np.float32)
    net = orbopt.LearnedPreconditioner(seed=3)
    net.train(X, y, epochs=1, batch=64)  # fixes the standardisation, moves the weights off the init
    loss, g = net.loss_and_grad(X, y)
    p = net.get_params()
    lref, gref = np_loss_and_grad(p.astype(np.float64), X.astype(np.float64), y.astype(np.float64))
    assert abs(loss - lref) <= 1e-4 * max(1.0, lref)
    assert np.abs(g - gref).max() <= 1e-4 * max(1e-3, np.abs(gref).max())
    # finite-difference check of the float64 restatement on a few weights
    for i in (3, 600, 5000, 8960):
        dp = np.zeros_like(p, dtype=np.float64)
        dp[i] = 1e-5
        lp = np_loss_and_grad(p + dp, X, y)[0]
        lm = np_loss_and_grad(p - dp, X, y)[0]
        assert abs((lp - lm) / 2e-5 - gref[i]) <= 1e-5 * max(1.0, abs(gref[i]))
    net.close()


def test_mlp_training_and_bf16_inference():
    rng = np.random.default_rng(8)
    X = rng.standard_normal((4000, 8)).astype(np.float32)
    y = (np.tanh(X[:, 0] * X[:, 1]) + 0.3 * X[:, 2] ** 2 - X[:, 7]).astype(np.float32)
    net = orbopt.LearnedPreconditioner(seed=1)
    hist = net.train(X, y, epochs=40, batch=256, learning_rate=3e-3)
    assert hist[-1] < 0.1 * hist[0]
    y32 = net.predict(X[:500], bf16=False)
    y16 = net.predict(X[:500], bf16=True)
    assert np.abs(y16 - y32).max() <= 0.05 * max(1.0, np.abs(y32).max())
    assert np.corrcoef(y32, y[:500])[0, 1] > 0.97
    p = net.get_params()
    net2 = orbopt.LearnedPreconditioner(seed=99)
    net2.set_params(p)
    assert np.array_equal(net2.predict(X[:100], bf16=False), y32[:100])
    net.close()
    net2.close()


def test_learned_preconditioner_cuts_macro_iterations():
    """The shipped preconditioner (trained by rerdmft_b200.precond_train on seeds 1000+) against
    plain ADAM on held-out systems: fewer macro-iterations in total, the same converged energies."""
    net = orbopt.load_default_preconditioner()
    tot = {"plain": 0, "learned": 0}
    for seed in range(1, 7):
        for nocc in (2, 3):
            e = {}
            for mode in tot:
                prob, eri = orbopt.problem_from_system(synth.functional_system(8, 32, seed, nocc=nocc))
                r = orbopt.run_full_optimization(prob, preconditioner=net if mode == "learned" else None)
                assert r["converged"]
                tot[mode] += r["macro_iterations"]
                e[mode] = r["energy"]
                prob.close()
            assert abs(e["learned"] - e["plain"]) <= 1e-8
    assert tot["learned"] <= 0.70 * tot["plain"], tot  # at least 30 % fewer macro-iterations
    net.close()


def _gnof_problem(n, nocc, coupling, seed, naux=24):
    from rerdmft_b200 import pnof

    f = synth.functional_system(n, naux, seed, nocc=nocc)
    gem = pnof.nonrel_geminals(n, nocc, coupling)
    occ0 = pnof.occupations_of(gem, coupling, np.full(nocc * (coupling - 1), np.pi / 4), 2 * n)
    two = pnof.full_two_rdm(pnof.FUNCTIONALS["GNOF"], gem, occ0, 2 * n)
    eri = mo.RiNonRelSpinMoEri.from_tensor(f["Bmo"], n)
    prob = orbopt.RotationProblem(eri, f["h"], occ0, two["two_rdm_h"], two["two_rdm_x"], two["pair_of"],
                                  two["two_rdm_l1"], two["two_rdm_l2"])
    return f, gem, prob, eri


def test_gnof_full_optimization_matches_reference_energy(ref_lib):
    """GNOF FULL_OPTIMIZATION (device ADAM orbital runs, host occupation steps from the device J/K):
    converged; the final energy is the reference's pnofElectronicEnergy at the final orbitals and
    occupations, and the device rotation problem's energy (generalized-Fock trace with the full two-RDM)
    is the same number; the learned preconditioner reaches the same energy."""
    from rerdmft_b200 import pnof

    n, nocc, coupling = 8, 2, 3
    f, gem, prob, eri = _gnof_problem(n, nocc, coupling, 6)
    r = pnof.run_pnof_optimization(prob, "GNOF", gem, coupling)
    assert r["converged"]
    u, hr, b = prob.state(with_tensor=True)
    H = np.zeros((2 * n, 2 * n))
    H[:n, :n] = hr
    H[n:, n:] = hr
    e_ref, _ = ref_lib.pnof_energy_nonrel("GNOF", gem, r["occupations"], b, n, H)
    assert abs(r["energy"] - e_ref) <= 1e-10 * max(1.0, abs(e_ref))
    assert abs(prob.energy() - e_ref) <= 1e-10 * max(1.0, abs(e_ref))
    assert np.abs(prob.gradient()).max() < 1e-3
    assert np.all(np.diff(r["history"][1:]) < 1e-7)  # macro-iteration energies do not rise
    prob.close()
    net = orbopt.load_default_preconditioner()
    f, gem, prob, eri = _gnof_problem(n, nocc, coupling, 6)
    rl = pnof.run_pnof_optimization(prob, "GNOF", gem, coupling, preconditioner=net)
    assert rl["converged"] and abs(rl["energy"] - r["energy"]) <= 1e-7
    prob.close()
    net.close()
