"""Orbital-rotation optimisation of the functional stage on the GPU, and its learned preconditioner.

* ``RotationProblem``        src/Full_opt/FullOptimization.cpp:1330-1548 (RotationProblem) with
                             ``run`` = AdamOptimizer::run, src/Utils/ADAM.cpp:140-213
* ``adam_default_options``   AdamOptions, src/Utils/ADAM.h:41-60
* ``run_full_optimization``  the orbital half of the FULL_OPTIMIZATION macro loop: repeated ADAM runs at
                             fixed occupations until the best energy changes by less than ``tol`` without
                             a restart request (m_noft_driver's rule, ADAM.h:205-209)
* ``LearnedPreconditioner``  no counterpart in the reference: an MLP predicting the diagonal orbital
                             Hessian (hartreeExchangeHessianElement(p,q,p,q)) from eight per-pair inputs;
                             its predictions rescale the ADAM pairs (rr_orbopt_set_scales)

The functional is a fixed-occupation hartree-exchange form (two_rdm_h, two_rdm_x and optionally the
pair terms pair_of / two_rdm_l1 / two_rdm_l2) over the nonrelativistic spin-orbital RI tensor
(``mo.RiNonRelSpinMoEri``) or the complex spinor tensor (``mo.RiMoEri``, X2C / 4c), as in the
reference's RI FULL_OPTIMIZATION.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib as L
from ._lib import RrError


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def adam_default_options() -> L.AdamOptions:
    o = L.AdamOptions()
    L.check(L.lib().rr_adam_default_options(ctypes.byref(o)))
    return o


class RotationProblem:
    """ADAM orbital-rotation problem on the GPU (RotationProblem<T, Eri>) for `eri`:

    * ``RiNonRelSpinMoEri`` (n spatial orbitals): h is the n x n spatial one-electron matrix in eri's
      MO basis; occupations 2n; two_rdm_h / two_rdm_x 2n x 2n; optional pair_of (2n) with
      two_rdm_l1 / two_rdm_l2 (2n x 2n).  Pairs adamPairIndices(2n), spin-twin averaged gradient.
    * ``RiMoEri`` (n spinors, complex): h complex n x n; occupations n; two-RDM factors n x n;
      optional pair_of (n) with l1 / l2; ``n_negative`` drops the pairs touching the first
      n_negative spinors (excludeNegative, FullOptimization.cpp:83-92).  Complex gradient and steps."""

    def __init__(self, eri, h, occupations, two_rdm_h, two_rdm_x, pair_of=None, two_rdm_l1=None, two_rdm_l2=None,
                 options: L.AdamOptions | None = None, n_negative: int = 0):
        n = eri.n
        self.complex = getattr(eri, "_kind", L.RR_MO_NONREL_SPIN) == L.RR_MO_COMPLEX
        d = n if self.complex else 2 * n
        h = np.ascontiguousarray(h, dtype=np.complex128) if self.complex else _d(h)
        if h.shape != (n, n):
            raise RrError(L.RR_ERR_ARG, "RotationProblem: h must be n x n in the tensor's MO basis")
        occ = _d(occupations)
        h2, x2 = _d(two_rdm_h), _d(two_rdm_x)
        if occ.shape != (d,) or h2.shape != (d, d) or x2.shape != (d, d):
            raise RrError(L.RR_ERR_ARG, "RotationProblem: occupations / two-RDMs must span the %d accessor orbitals" % d)
        if n_negative and not self.complex:
            raise RrError(L.RR_ERR_UNSUPPORTED, "RotationProblem: n_negative needs the complex RiMoEri tensor")
        po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
        l1 = None if po is None else _d(two_rdm_l1)
        l2 = None if po is None else _d(two_rdm_l2)
        self.handle = ctypes.c_void_p()
        L.check(L.lib().rr_orbopt_create(eri.handle, h.ctypes.data, occ.ctypes.data, h2.ctypes.data, x2.ctypes.data,
                                         None if po is None else po.ctypes.data,
                                         None if po is None else l1.ctypes.data,
                                         None if po is None else l2.ctypes.data,
                                         None if options is None else ctypes.byref(options), ctypes.byref(self.handle)))
        if n_negative:
            L.check(L.lib().rr_orbopt_exclude_negative(self.handle, int(n_negative)))
        self.n, self.d, self.n_negative = n, d, int(n_negative)
        pq = [(pp, qq) for pp in range(d) for qq in range(pp) if pp >= self.n_negative and qq >= self.n_negative]
        self.n_pairs = len(pq)
        self.pairs = np.array(pq, dtype=int).reshape(-1, 2)
        if self.complex:
            self.cross_spin = np.zeros(self.n_pairs, dtype=bool)
        else:
            self.cross_spin = (self.pairs[:, 0] >= n) != (self.pairs[:, 1] >= n)

    @property
    def _dt(self):
        return np.complex128 if self.complex else np.float64

    def close(self):
        if self.handle and self.handle.value:
            L.lib().rr_orbopt_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def run(self) -> dict:
        r = L.AdamResult()
        L.check(L.lib().rr_orbopt_run(self.handle, ctypes.byref(r)))
        return r.as_dict()

    def energy(self) -> float:
        e = ctypes.c_double()
        L.check(L.lib().rr_orbopt_energy(self.handle, ctypes.byref(e)))
        return e.value

    def gradient(self) -> np.ndarray:
        g = np.empty(self.n_pairs, dtype=self._dt)
        L.check(L.lib().rr_orbopt_gradient(self.handle, g.ctypes.data))
        return g

    def hessian_diagonal(self) -> np.ndarray:
        """Per-pair diagonal Hessian; the joint [t; y] diagonal (2 n_pairs) for a complex problem."""
        h = np.empty(2 * self.n_pairs if self.complex else self.n_pairs)
        L.check(L.lib().rr_orbopt_hessian_diagonal(self.handle, h.ctypes.data))
        return h

    def features(self) -> np.ndarray:
        f = np.empty((self.n_pairs, 8), dtype=np.float32)
        L.check(L.lib().rr_orbopt_features(self.handle, f.ctypes.data))
        return f

    def set_scales(self, scales=None):
        if scales is None:
            L.check(L.lib().rr_orbopt_set_scales(self.handle, None))
            return
        s = _d(scales)
        if s.shape != (self.n_pairs,):
            raise RrError(L.RR_ERR_ARG, "RotationProblem.set_scales: one scale per pair")
        L.check(L.lib().rr_orbopt_set_scales(self.handle, s.ctypes.data))

    def set_functional(self, occupations, two_rdm_h, two_rdm_x, pair_of=None, two_rdm_l1=None, two_rdm_l2=None):
        """New occupations and two-RDM factors for the next runs (orbitals, ADAM state and scales kept)."""
        occ = _d(occupations)
        h2, x2 = _d(two_rdm_h), _d(two_rdm_x)
        if occ.shape != (self.d,) or h2.shape != (self.d, self.d) or x2.shape != (self.d, self.d):
            raise RrError(L.RR_ERR_ARG, "RotationProblem.set_functional: shapes differ from the problem's")
        po = None if pair_of is None else np.ascontiguousarray(pair_of, dtype=np.int64)
        l1 = None if po is None else _d(two_rdm_l1)
        l2 = None if po is None else _d(two_rdm_l2)
        L.check(L.lib().rr_orbopt_set_functional(self.handle, occ.ctypes.data, h2.ctypes.data, x2.ctypes.data,
                                                 None if po is None else po.ctypes.data,
                                                 None if po is None else l1.ctypes.data,
                                                 None if po is None else l2.ctypes.data))

    def jk(self):
        """J_ij = eri(i,j,i,j), K_ij = eri(i,j,j,i) of the current tensor (d x d)."""
        J = np.empty((self.d, self.d), dtype=self._dt)
        K = np.empty((self.d, self.d), dtype=self._dt)
        L.check(L.lib().rr_orbopt_jk(self.handle, J.ctypes.data, K.ctypes.data))
        return J, K

    def jk_and_h_diag(self):
        """(real J, real K, the diagonal of the current one-electron matrix over the d accessor orbitals)."""
        J, K = self.jk()
        _, h, _ = self.state()
        hd = np.real(np.diag(h))
        if not self.complex:
            hd = np.concatenate([hd, hd])
        return np.real(J), np.real(K), hd

    def state(self, with_tensor: bool = False):
        """(accumulated rotation, rotated h, rotated MO tensor or None)."""
        u = np.empty((self.n, self.n), dtype=self._dt)
        h = np.empty((self.n, self.n), dtype=self._dt)
        naux = ctypes.c_int64()
        L.check(L.lib().rr_orbopt_info(self.handle, None, None, ctypes.byref(naux)))
        b = np.empty((naux.value, self.n * self.n), dtype=self._dt) if with_tensor else None
        L.check(L.lib().rr_orbopt_state(self.handle, u.ctypes.data, h.ctypes.data, None if b is None else b.ctypes.data))
        return u, h, b


def hessian_scales(problem: RotationProblem, hdiag, clip: float = 16.0, quantile: float = 0.5) -> np.ndarray:
    """Scales from a (predicted or exact) diagonal Hessian: |H| / (the `quantile` of |H| over the
    same-spin pairs, the median by default), clipped to [1/clip, 1], so pairs softer than that
    reference take up to sqrt(clip) times larger rotations and none is slowed down (shrinking the stiff
    pairs as well cost more iterations than it saved on the synthetic functional-stage problems);
    cross-spin pairs (zero gradient) keep 1."""
    h = np.abs(np.asarray(hdiag, dtype=float))
    if h.shape[0] == 2 * problem.n_pairs and problem.complex:  # joint [t; y] diagonal: one scale per pair
        h = 0.5 * (h[: problem.n_pairs] + h[problem.n_pairs:])
    same = ~problem.cross_spin
    med = np.quantile(h[same], quantile) if same.any() else 1.0
    if not med > 0:
        med = 1.0
    s = np.clip(h / med, 1.0 / clip, 1.0)
    s[problem.cross_spin] = 1.0
    return s


class LearnedPreconditioner:
    """The 8 -> 64 -> 64 -> 64 -> 1 MLP (librr_ri rr_mlp_*) mapping rr_orbopt_features to
    log |H_diag|; trained in FP32, BF16 inference."""

    N_PARAMS = 8961
    N_NORM = 18

    def __init__(self, seed: int = 0):
        self.handle = ctypes.c_void_p()
        L.check(L.lib().rr_mlp_create(ctypes.c_uint64(seed), ctypes.byref(self.handle)))

    def close(self):
        if self.handle and self.handle.value:
            L.lib().rr_mlp_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def labels(hdiag) -> np.ndarray:
        return np.log(np.maximum(np.abs(np.asarray(hdiag, dtype=float)), 1e-8)).astype(np.float32)

    def train(self, X, y, epochs: int = 60, batch: int = 256, learning_rate: float = 2e-3, seed: int = 1):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        hist = np.empty(epochs, dtype=np.float32)
        L.check(L.lib().rr_mlp_train(self.handle, X.ctypes.data, y.ctypes.data, X.shape[0], epochs, batch,
                                     ctypes.c_float(learning_rate), ctypes.c_uint64(seed), hist.ctypes.data))
        return hist

    def predict(self, X, bf16: bool = True) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.empty(X.shape[0], dtype=np.float32)
        L.check(L.lib().rr_mlp_predict(self.handle, X.ctypes.data, X.shape[0], int(bf16), y.ctypes.data))
        return y

    def loss_and_grad(self, X, y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.empty(self.N_PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        L.check(L.lib().rr_mlp_loss_and_grad(self.handle, X.ctypes.data, y.ctypes.data, X.shape[0], ctypes.byref(loss),
                                             g.ctypes.data))
        return float(loss.value), g

    def get_params(self) -> np.ndarray:
        p = np.empty(self.N_PARAMS + self.N_NORM, dtype=np.float32)
        L.check(L.lib().rr_mlp_get_params(self.handle, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (self.N_PARAMS + self.N_NORM,):
            raise RrError(L.RR_ERR_ARG, "LearnedPreconditioner.set_params: wrong parameter count")
        L.check(L.lib().rr_mlp_set_params(self.handle, p.ctypes.data))

    def scales(self, problem: RotationProblem, clip: float = 16.0, bf16: bool = True,
               quantile: float = 0.9) -> np.ndarray:
        return hessian_scales(problem, np.exp(self.predict(problem.features(), bf16=bf16)), clip, quantile)


def run_full_optimization(problem: RotationProblem, tol: float = 1e-8, max_macro: int = 400,
                          preconditioner: LearnedPreconditioner | None = None, exact_hessian: bool = False,
                          clip: float = 16.0, polish: bool = True, quantile: float = 0.9) -> dict:
    """Macro loop of ADAM runs at fixed occupations (the orbital half of FULL_OPTIMIZATION): stop when
    two successive runs' best energies differ by less than `tol` and the optimiser asked for no
    restart.  With a preconditioner (or exact_hessian) the pair scales are refreshed before every
    run from the current orbitals; with `polish` the plain method then continues from the
    preconditioned result until it meets the same rule, so plain ADAM settles the converged energy
    (the rescaled runs only move the start).  Iterations of both phases are counted.  The scales use the
    90th percentile of the (predicted) curvature as reference (hessian_scales): on the synthetic
    functional-stage problems the median reference saved 19 % of the macro-iterations, the 90th
    percentile 40 % (learned) and 44 % (exact Hessian)."""
    t0 = time.perf_counter()
    steps = 0
    history = []
    scaled = preconditioner is not None or exact_hessian
    phases = ["scaled", "plain"] if scaled and polish else (["scaled"] if scaled else ["plain"])
    m = 0
    converged = False
    scaled_macro = 0
    e_prev = None
    for phase in phases:
        if phase == "plain":
            problem.set_scales(None)
        # the plain rule compares with the previous run's best energy, whichever phase ran it
        converged = False
        while m < max_macro:
            m += 1
            if phase == "scaled":
                scaled_macro += 1
                if preconditioner is not None:
                    problem.set_scales(preconditioner.scales(problem, clip, quantile=quantile))
                else:
                    problem.set_scales(hessian_scales(problem, problem.hessian_diagonal(), clip, quantile))
            r = problem.run()
            steps += r["iterations"]
            history.append(r["energy_best"])
            if e_prev is not None and abs(r["energy_best"] - e_prev) < tol and not r["restart_requested"]:
                converged = True
                break
            e_prev = r["energy_best"]
    return dict(macro_iterations=m, adam_steps=steps, energy=history[-1], converged=converged,
                scaled_macro_iterations=scaled_macro, seconds=time.perf_counter() - t0, history=np.array(history))


def muller_functional(occ_spatial):
    """Spin-orbital occupations and the Mueller-type two-RDM factors two_rdm_h = n_p n_q,
    two_rdm_x = sqrt(n_p n_q) of a fixed set of spatial occupations (a JK-only functional)."""
    n = np.concatenate([occ_spatial, occ_spatial]).astype(float)
    return n, np.outer(n, n), np.sqrt(np.outer(n, n))


def training_data(problems, samples_per_problem: int = 4, runs_between: int = 2, rng=None):
    """(features, labels) from each problem at several points of its plain-ADAM path: features from
    rr_orbopt_features, labels log |hartreeExchangeHessianElement(p,q,p,q)|, same-spin pairs only."""
    rng = rng if rng is not None else np.random.default_rng(0)
    Xs, ys = [], []
    for prob in problems:
        prob.set_scales(None)
        for k in range(samples_per_problem):
            f = prob.features()
            hd = prob.hessian_diagonal()
            keep = ~prob.cross_spin
            Xs.append(f[keep])
            ys.append(LearnedPreconditioner.labels(hd[keep]))
            for _ in range(runs_between):
                prob.run()
    return np.concatenate(Xs), np.concatenate(ys)


PARAMS_FILE = __import__("pathlib").Path(__file__).resolve().parent / "data" / "precond_mlp.npy"


def problem_from_system(sysd: dict, options: L.AdamOptions | None = None):
    """(RotationProblem, MO tensor) for a dict of rerdmft_b200.synth.functional_system's form (or
    functional_system_complex's, which carries the complex spinor tensor and n_negative)."""
    from .mo import RiMoEri, RiNonRelSpinMoEri

    extra = {k: sysd[k] for k in ("pair_of", "two_rdm_l1", "two_rdm_l2") if k in sysd}
    if np.iscomplexobj(sysd["Bmo"]):
        eri = RiMoEri.from_tensor(sysd["Bmo"], sysd["n"])
        extra["n_negative"] = sysd.get("n_negative", 0)
    else:
        eri = RiNonRelSpinMoEri.from_tensor(sysd["Bmo"], sysd["ns"])
    prob = RotationProblem(eri, sysd["h"], sysd["occupations"], sysd["two_rdm_h"], sysd["two_rdm_x"],
                           options=options, **extra)
    return prob, eri


def load_default_preconditioner() -> LearnedPreconditioner:
    """The preconditioner trained by ``python -m rerdmft_b200.precond_train`` (shipped parameters)."""
    net = LearnedPreconditioner(seed=0)
    net.set_params(np.load(PARAMS_FILE))
    return net
