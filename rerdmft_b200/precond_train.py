"""Trains the learned orbital-rotation preconditioner on the GPU and writes its parameters.

    python -m rerdmft_b200.precond_train [--out rerdmft_b200/data/precond_mlp.npy] [--systems 200]

Data: `--systems` seeded synthetic functional-stage systems (rerdmft_b200.synth.functional_system,
6 to 12 spatial orbitals, naux = 4 ns, 2 to 4 strongly occupied orbitals, every third one with pair
terms) plus eight larger ones (20 to 80 spatial orbitals); each contributes the same-spin pairs at
several points of its plain-ADAM path, features from
rr_orbopt_features and labels log |hartreeExchangeHessianElement(p,q,p,q)| from
rr_orbopt_hessian_diagonal.  Training: the library's FP32 kernels, mini-batch Adam, 60 epochs.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import orbopt, synth


LARGE_SIZES = (20, 24, 30, 40, 40, 60, 60, 80)


def build_dataset(n_systems: int, first_seed: int = 1000):
    probs = []
    for k in range(n_systems):
        seed = first_seed + k
        ns = 6 + k % 7
        s = synth.functional_system(ns, 4 * ns, seed, nocc=2 + k % 3, with_pairs=(k % 3 == 0))
        probs.append(orbopt.problem_from_system(s))
    X1, y1 = orbopt.training_data([p for p, _ in probs], samples_per_problem=4, runs_between=3)
    for p, _ in probs:
        p.close()
    probs = [orbopt.problem_from_system(synth.functional_system(ns, 4 * ns, 5000 + k, nocc=2 + k % 3))
             for k, ns in enumerate(LARGE_SIZES)]
    X2, y2 = orbopt.training_data([p for p, _ in probs], samples_per_problem=3, runs_between=4)
    for p, _ in probs:
        p.close()
    return np.concatenate([X1, X2]), np.concatenate([y1, y2])


def train(n_systems: int = 200, epochs: int = 60, seed: int = 0):
    t0 = time.perf_counter()
    X, y = build_dataset(n_systems)
    t1 = time.perf_counter()
    net = orbopt.LearnedPreconditioner(seed=seed)
    hist = net.train(X, y, epochs=epochs, batch=256, learning_rate=2e-3)
    t2 = time.perf_counter()
    return net, dict(pairs=int(X.shape[0]), data_seconds=t1 - t0, train_seconds=t2 - t1,
                     loss_first=float(hist[0]), loss_last=float(hist[-1]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(orbopt.PARAMS_FILE))
    ap.add_argument("--systems", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=60)
    args = ap.parse_args()
    net, info = train(args.systems, args.epochs)
    np.save(args.out, net.get_params())
    print(info)


if __name__ == "__main__":
    main()
