"""Pins of the integral oracle (oracle/integrals_oracle.py) and of the host basis code (rerdmft_b200.basis),
no GPU: the Boys function against quadrature, s-type integrals against their closed form, p and d functions
against finite differences of s functions in the centre coordinates, and the RI Hartree-Fock energy of
LiH / 6-31G from these integrals against the value the reference printed with libcint's integrals
(examples/reference.yaml, stored in tests/golden/lih_631g*.npz)."""
import math

import numpy as np
import pytest
from scipy import integrate
from scipy.special import erf

import molecules
from oracle import integrals_oracle as io
from oracle import ri_oracle as ro
from rerdmft_b200 import basis as bs


def test_boys_against_quadrature():
    for T in (0.0, 1e-10, 0.3, 5.0, 20.0, 35.9, 36.1, 60.0, 200.0):
        F = io.boys(12, np.array(T))
        for n in range(13):
            ref = integrate.quad(lambda t: t ** (2 * n) * math.exp(-T * t * t), 0.0, 1.0, epsabs=0, epsrel=1e-13,
                                 limit=200)[0]
            assert abs(F[n] - ref) <= 1e-12 * ref, (T, n)


def _prim(center, l, a):
    """A primitive whose monomial carries coefficient 1 (the libcint factor divided out)."""
    s = io._Sh(center, l, [a], [1.0])
    s.k = np.array([1.0])
    return s


def test_s_type_closed_form():
    rng = np.random.default_rng(3)
    for _ in range(5):
        A, B, C = rng.uniform(-1.5, 1.5, (3, 3))
        a, b, c = rng.uniform(0.2, 3.0, 3)
        v = io.eri3_block(_prim(A, 0, a), _prim(B, 0, b), _prim(C, 0, c))[0, 0, 0]
        p = a + b
        P = (a * A + b * B) / p
        T = p * c / (p + c) * float((P - C) @ (P - C))
        F0 = 0.5 * math.sqrt(math.pi / T) * erf(math.sqrt(T))
        ref = 2 * math.pi ** 2.5 / (p * c * math.sqrt(p + c)) * math.exp(-a * b / p * float((A - B) @ (A - B))) * F0
        assert abs(v - ref) <= 1e-13 * abs(ref)


def _shift(x, d, h):
    y = np.array(x, dtype=np.float64)
    y[d] += h
    return y


@pytest.mark.parametrize("which", ["a", "b", "c"])
def test_p_and_d_from_center_derivatives(which):
    """x_A exp(-a r_A^2) = (1 / 2a) d/dA_x exp(-a r_A^2); x_A y_A exp = (1 / 4a^2) d2/dA_x dA_y exp;
    x_A^2 exp = (d2/dA_x^2 exp + 2a exp) / (4a^2), for the bra's first or second factor and the aux factor."""
    rng = np.random.default_rng({"a": 1, "b": 2, "c": 4}[which])
    A, B, C = rng.uniform(-1.2, 1.2, (3, 3))
    a, b, c = rng.uniform(0.4, 2.0, 3)
    cen = {"a": A, "b": B, "c": C}
    ex = {"a": a, "b": b, "c": c}[which]

    def s_val(center):
        shells = {"a": _prim(A, 0, a), "b": _prim(B, 0, b), "c": _prim(C, 0, c)}
        shells[which] = _prim(center, 0, ex)
        return io.eri3_block(shells["a"], shells["b"], shells["c"])[0, 0, 0]

    def block(l):
        shells = {"a": _prim(A, 0, a), "b": _prim(B, 0, b), "c": _prim(C, 0, c)}
        shells[which] = _prim(cen[which], l, ex)
        blk = io.eri3_block(shells["a"], shells["b"], shells["c"])
        return blk.reshape(-1)

    X = cen[which]
    h = 1e-4
    p = block(1)  # x, y, z
    for d in range(3):
        fd = (s_val(_shift(X, d, h)) - s_val(_shift(X, d, -h))) / (2 * h) / (2 * ex)
        assert abs(p[d] - fd) <= 1e-7 * max(abs(fd), 1e-3), (d, p[d], fd)
    dd = block(2)  # xx, xy, xz, yy, yz, zz
    h2 = 1e-3
    s0 = s_val(X)
    comps = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    for k, (d1, d2) in enumerate(comps):
        if d1 == d2:
            sec = (s_val(_shift(X, d1, h2)) - 2 * s0 + s_val(_shift(X, d1, -h2))) / (h2 * h2)
            fd = (sec + 2 * ex * s0) / (4 * ex * ex)
        else:
            pp = s_val(_shift(_shift(X, d1, h2), d2, h2))
            pm = s_val(_shift(_shift(X, d1, h2), d2, -h2))
            mp = s_val(_shift(_shift(X, d1, -h2), d2, h2))
            mm = s_val(_shift(_shift(X, d1, -h2), d2, -h2))
            fd = (pp - pm - mp + mm) / (4 * h2 * h2) / (4 * ex * ex)
        assert abs(dd[k] - fd) <= 1e-5 * max(abs(fd), 1e-3), (k, dd[k], fd)


def test_metric_is_the_three_centre_sum_with_a_constant():
    """(P|Q) = (P 1|Q): the metric's unit bra factor against a wide s function's limit."""
    rng = np.random.default_rng(7)
    A, C = rng.uniform(-1, 1, (2, 3))
    for la, lc in ((0, 0), (1, 2), (2, 1)):
        Psh, Qsh = _prim(A, la, 0.9), _prim(C, lc, 1.3)
        exact = io.eri3_block(Psh, io._unit_s(A), Qsh)[:, 0, :]
        wide = io.eri3_block(Psh, _prim(A, 0, 1e-9), Qsh)[:, 0, :]
        assert np.abs(exact - wide).max() <= 1e-7 * np.abs(exact).max()


def test_normalisation_and_shells():
    m = molecules.load("lih_631g")
    S = io.overlap_matrix(m["basis"])
    assert np.abs(np.diag(S) - 1.0).max() < 1e-14
    assert bs.group_into_shells(m["basis"]) == [(0, 1), (1, 1), (2, 3), (5, 1), (6, 3), (9, 1), (10, 1)]
    Ma = io.aux_metric(m["aux"])
    assert np.abs(np.diag(Ma) - np.diag(Ma)).max() == 0.0
    # every aux function: one primitive, unit self-overlap after normalisation
    Sa = io.overlap_matrix(m["aux"])
    assert np.abs(np.diag(Sa) - 1.0).max() < 1e-13


def test_auxiliary_basis_recipe():
    m = molecules.load("lih_631g")
    aux = m["aux"]
    assert len(aux) == 106
    shells = bs.group_into_shells(aux)
    # per centre, the cluster exponents decrease and the angular momenta of each cluster start at 0
    last = {}
    for first, cnt in shells:
        f = aux[first]
        key = (f.x, f.y, f.z)
        if f.l == 0:
            assert key not in last or f.exponents[0] < last[key]
            last[key] = f.exponents[0]
    auto = bs.build_auto_auxiliary_basis(m["basis"], "AUTO")
    assert 0 < len(auto) < len(aux)


def _ri_hf(m, guesses):
    orb, aux = m["basis"], m["aux"]
    S = io.overlap_matrix(orb)
    ch = [(bs.atomic_number(a.symbol), (a.x, a.y, a.z)) for a in m["geometry"]]
    h = io.kinetic_matrix(orb) + io.nuclear_attraction_matrix(orb, ch)
    X = ro.canonical_orthogonalize(S, 1e-6)
    Mx = ro.canonical_orthogonalize(io.aux_metric(aux), 1e-10)
    B = Mx.T @ io.three_center_raw(orb, aux)
    enuc = bs.nuclear_repulsion(m["geometry"])
    out = []
    for D0 in guesses(h, X):
        r = ro.nonrel_scf(dict(h=h, B=B, S=S, X=X, n_electrons=m["nelec"], D0=D0), max_iter=200)
        if r["converged"]:
            out.append(r["energy"] + enuc)
    return out, Mx.shape


def test_lih_ri_hf_energy_matches_reference():
    m = molecules.load("lih_631g")
    e, mshape = _ri_hf(m, lambda h, X: [molecules.core_guess(h, X, m["nelec"] // 2)])
    assert mshape == (106, 104)  # the metric's LOWGEN drops two near-dependent directions at 1e-10
    assert abs(e[0] - m["e_hf_ri"]) < 1e-8, e[0] - m["e_hf_ri"]
    assert abs(e[0] - m["e_hf_dense"]) > 1e-5  # the RI value, not the dense one


def test_lih_stretched_lowest_state_matches_reference():
    m = molecules.load("lih_631g_5a")
    e, _ = _ri_hf(m, lambda h, X: molecules.random_guesses(X, m["nelec"] // 2, seed=0, count=12))
    assert abs(min(e) - m["e_hf_ri"]) < m["tolerance"], min(e) - m["e_hf_ri"]


@pytest.mark.parametrize("l", range(7))
def test_spherical_blocks(l):
    """Each block (src/Utils/SphericalTransform.cpp:60-130) spans the Laplacian's null space on degree-l
    monomials and is orthonormal in the overlap of the normalised Cartesian components."""
    blk = bs.cartesian_to_spherical_block(l)
    comps = bs.cartesian_components(l)
    assert blk.shape == (len(comps), 2 * l + 1)
    raw = np.array([[bs.cartesian_self_overlap_pair(l, a, b) for b in comps] for a in comps])
    d = 1.0 / np.sqrt(np.diag(raw))
    s_norm = raw * d[:, None] * d[None, :]
    assert np.abs(blk.T @ s_norm @ blk - np.eye(2 * l + 1)).max() < 1e-12
    if l >= 2:
        assert np.abs(bs._laplacian(l) @ blk).max() < 1e-12 * max(1.0, np.abs(blk).max())


def test_spherical_transform_of_a_basis():
    m = molecules.load("water_ccpvdz")
    T, shells = bs.build_spherical_transform(m["basis"])
    assert T.shape == (25, 24) and len(shells) == 12
    S = io.overlap_matrix(m["basis"])
    Ss = T.T @ S @ T
    assert np.abs(np.diag(Ss) - 1.0).max() < 1e-12  # the transformed functions stay normalised
