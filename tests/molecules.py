"""Molecular test systems from the fixtures written by tests/golden/make_integrals_golden.py (test helper)."""
from __future__ import annotations

import numpy as np

from rerdmft_b200 import basis as bs

from conftest import golden


def load(name: str, aux_kind: str = "PAUTO") -> dict:
    """geometry (bohr), the normalised orbital basis, the normalised automatic aux basis, nelec and the
    reference energies stored with the fixture."""
    z = golden(name)
    sets = bs.basis_set_from_arrays(z["shell_element"], z["shell_l"], z["shell_nprim"], z["exponents"],
                                    z["coefficients"])
    geo = [bs.Atom(str(s), *map(float, xyz)) for s, xyz in zip(z["atom_symbol"], z["atom_xyz"])]
    orb = bs.build_molecular_basis(geo, sets)
    bs.normalize_cartesian_basis(orb)
    aux = bs.build_auto_auxiliary_basis(orb, aux_kind)
    bs.normalize_cartesian_basis(aux)
    out = dict(geometry=geo, basis=orb, aux=aux, nelec=int(z["nelec"]))
    for k in ("e_hf_ri", "e_hf_dense", "tolerance"):
        if k in z:
            out[k] = float(z[k])
    return out


def core_guess(h: np.ndarray, X: np.ndarray, nocc: int) -> np.ndarray:
    """Density of the lowest nocc eigenvectors of X^T h X (doubly occupied)."""
    w, u = np.linalg.eigh(X.T @ h @ X)
    c = X @ u[:, :nocc]
    return 2.0 * c @ c.T


def random_guesses(X: np.ndarray, nocc: int, seed: int, count: int) -> list:
    """Densities of `count` seeded random orthonormal occupied sets (searching the SCF solutions)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        q = np.linalg.qr(rng.standard_normal((X.shape[1], X.shape[1])))[0][:, :nocc]
        c = X @ q
        out.append(2.0 * c @ c.T)
    return out
