"""The device integral engine (rr_int_aux_metric, rr_int_three_center_raw, rr_ri_create_basis) against the
oracle (oracle/integrals_oracle.py, itself pinned by tests/test_integrals_oracle.py), and end to end: the RI
Hartree-Fock energy of LiH / 6-31G from device integrals and the device SCF loop against the value the
reference printed (libcint integrals, examples/reference.yaml)."""

import numpy as np
import pytest

import molecules
from oracle import integrals_oracle as io
from oracle import ri_oracle as ro
from rerdmft_b200 import _lib as L
from rerdmft_b200 import basis as bs
from rerdmft_b200 import integrals as gi
from rerdmft_b200 import ri, scf

pytestmark = pytest.mark.gpu


def _close(a, b, rel=1e-12):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max()
    assert err <= rel * scale, (err, scale)


def test_boys_device_against_oracle():
    T = np.concatenate([[0.0, 1e-14, 1e-9], np.logspace(-6, 2.6, 300), [35.999, 36.0, 36.001]])
    nmax = 18
    out = np.empty((T.size, nmax + 1))
    L.check(L.lib().rr_test_boys(T.ctypes.data, T.size, nmax, out.ctypes.data))
    ref = io.boys(nmax, T).T
    rel = np.abs(out - ref) / np.abs(ref)
    i, n = np.unravel_index(rel.argmax(), rel.shape)
    assert rel.max() < 2e-13, (rel.max(), T[i], n)


@pytest.mark.parametrize("name", ["lih_631g", "water_ccpvdz"])
def test_metric_and_raw_against_oracle(name):
    m = molecules.load(name)
    _close(gi.auxMetric(m["aux"]), io.aux_metric(m["aux"]))
    _close(gi.threeCenterIntegralsRaw(m["basis"], m["aux"]), io.three_center_raw(m["basis"], m["aux"]))


def test_co_ccpvdz_every_aux_angular_momentum():
    """CO / cc-pVDZ with one aux shell of every angular momentum present (s .. f) per centre."""
    m = molecules.load("co_ccpvdz")
    aux = m["aux"]
    keep, seen = [], set()
    for first, cnt in bs.group_into_shells(aux):
        f = aux[first]
        key = (f.x, f.y, f.z, f.l)
        if key not in seen:
            seen.add(key)
            keep.extend(aux[first:first + cnt])
    assert {f.l for f in keep} == {0, 1, 2, 3}
    _close(gi.auxMetric(keep), io.aux_metric(keep))
    _close(gi.threeCenterIntegralsRaw(m["basis"], keep), io.three_center_raw(m["basis"], keep))


def _random_shell(rng, l, nprim, center):
    ex = sorted(rng.uniform(0.15, 6.0, nprim), reverse=True)
    co = list(rng.uniform(0.2, 1.0, nprim))
    return [bs.BasisFunction("X", *center, l, c, list(ex), list(co)) for c in bs.cartesian_components(l)]


def test_high_angular_momentum_and_ragged_layouts():
    """Orbital shells up to f and aux shells up to g at random centres (L up to 10), normalised; then the
    same functions with one shell split (non-proportional coefficients) and another permuted, so they are
    evaluated one function at a time."""
    rng = np.random.default_rng(11)
    cen = rng.uniform(-1.5, 1.5, (3, 3))
    orb = _random_shell(rng, 3, 2, cen[0]) + _random_shell(rng, 1, 3, cen[1]) + _random_shell(rng, 2, 1, cen[2])
    aux = _random_shell(rng, 3, 1, cen[1]) + _random_shell(rng, 0, 1, cen[0]) + _random_shell(rng, 4, 1, cen[2])
    bs.normalize_cartesian_basis(orb)
    bs.normalize_cartesian_basis(aux)
    _close(gi.auxMetric(aux), io.aux_metric(aux))
    raw = gi.threeCenterIntegralsRaw(orb, aux)
    _close(raw, io.three_center_raw(orb, aux))
    # ragged: perturb one component's coefficients (no longer proportional), permute the p shell
    rag = [bs.BasisFunction(f.element, f.x, f.y, f.z, f.l, f.cartesian, list(f.exponents), list(f.coefficients))
           for f in orb]
    rag[1].coefficients = [c * (1.0 + 0.1 * k) for k, c in enumerate(rag[1].coefficients)]
    rag[10], rag[12] = rag[12], rag[10]
    _close(gi.threeCenterIntegralsRaw(rag, aux), io.three_center_raw(rag, aux))


def test_invalid_basis_is_rejected():
    f = bs.BasisFunction("X", 0.0, 0.0, 0.0, 7, (7, 0, 0), [1.0], [1.0])
    with pytest.raises(L.RrError) as e:
        gi.auxMetric([f])
    assert e.value.code == L.RR_ERR_ARG
    g = bs.BasisFunction("X", 0.0, 0.0, 0.0, 0, (0, 0, 0), [-1.0], [1.0])
    with pytest.raises(L.RrError) as e:
        gi.auxMetric([g])
    assert e.value.code == L.RR_ERR_ARG


def _one_electron(m):
    orb = m["basis"]
    S = io.overlap_matrix(orb)
    ch = [(bs.atomic_number(a.symbol), (a.x, a.y, a.z)) for a in m["geometry"]]
    h = io.kinetic_matrix(orb) + io.nuclear_attraction_matrix(orb, ch)
    return S, h, ro.canonical_orthogonalize(S, 1e-6)


def _device_source(m, S, X):
    store, rep = gi.store_from_basis(m["basis"], m["aux"], 1e-10)
    return ri.RiNonRelEriSource(len(m["basis"]), None, X, S, store=store), rep


def test_store_from_basis_fock_matches_oracle():
    """The resident tensor built on the device from the basis sets gives the Fock matrix of the oracle's
    B = X_metric^T raw (an RI Fock build is invariant to the metric's orthogonalisation)."""
    m = molecules.load("water_ccpvdz")
    S, h, X = _one_electron(m)
    src, rep = _device_source(m, S, X)
    Mx = ro.canonical_orthogonalize(io.aux_metric(m["aux"]), 1e-10)
    assert rep["n_kept"] == Mx.shape[1]
    B = Mx.T @ io.three_center_raw(m["basis"], m["aux"])
    D = molecules.core_guess(h, X, m["nelec"] // 2)
    F = ri.nonRelFockMatrix(h, src, D)
    Fref = ro.nonrel_fock(h, B, D, S, X)
    assert np.abs(F - Fref).max() < 1e-10


def test_lih_ri_hf_energy_from_device_integrals():
    m = molecules.load("lih_631g")
    S, h, X = _one_electron(m)
    src, rep = _device_source(m, S, X)
    assert (rep["n_kept"], rep["n_dropped"]) == (104, 2)
    D0 = molecules.core_guess(h, X, m["nelec"] // 2)
    r = scf.runNonRelativisticHartreeFock(src, h, X, D0, m["nelec"])
    e = r["energy"] + bs.nuclear_repulsion(m["geometry"])
    assert r["converged"]
    assert abs(e - m["e_hf_ri"]) < 1e-8, e - m["e_hf_ri"]


def test_lih_stretched_lowest_state_from_device_integrals():
    m = molecules.load("lih_631g_5a")
    S, h, X = _one_electron(m)
    src, _ = _device_source(m, S, X)
    es = []
    for D0 in molecules.random_guesses(X, m["nelec"] // 2, seed=0, count=12):
        r = scf.runNonRelativisticHartreeFock(src, h, X, D0, m["nelec"], max_iterations=200)
        if r["converged"]:
            es.append(r["energy"] + bs.nuclear_repulsion(m["geometry"]))
    assert abs(min(es) - m["e_hf_ri"]) < m["tolerance"], min(es) - m["e_hf_ri"]


def test_device_outputs_stay_on_device():
    torch = pytest.importorskip("torch")
    m = molecules.load("lih_631g")
    M = gi.auxMetric(m["aux"], device=True)
    raw = gi.threeCenterIntegralsRaw(m["basis"], m["aux"], device=True)
    assert M.is_cuda and raw.is_cuda
    _close(M.cpu().numpy(), io.aux_metric(m["aux"]))
    _close(raw.cpu().numpy(), io.three_center_raw(m["basis"], m["aux"]))
    del torch


def test_spherical_store_from_basis():
    """rr_ri_create_basis with the Cartesian-to-spherical transform (the reference's CARTESIAN FALSE and
    relativistic large-component basis): the Fock matrix of the device store against the oracle's
    t^T B^P t of the restated integrals."""
    m = molecules.load("water_ccpvdz")
    T, _ = bs.build_spherical_transform(m["basis"])
    S = io.overlap_matrix(m["basis"])
    ch = [(bs.atomic_number(a.symbol), (a.x, a.y, a.z)) for a in m["geometry"]]
    h = io.kinetic_matrix(m["basis"]) + io.nuclear_attraction_matrix(m["basis"], ch)
    Ss, hs = T.T @ S @ T, T.T @ h @ T
    Xs = ro.canonical_orthogonalize(Ss, 1e-6)
    store, rep = gi.store_from_basis(m["basis"], m["aux"], 1e-10, t=T)
    ns = T.shape[1]
    src = ri.RiNonRelEriSource(ns, None, Xs, Ss, store=store)
    Mx = ro.canonical_orthogonalize(io.aux_metric(m["aux"]), 1e-10)
    B = ro.transform_ao_legs(Mx.T @ io.three_center_raw(m["basis"], m["aux"]), len(m["basis"]), T)
    D = molecules.core_guess(hs, Xs, m["nelec"] // 2)
    F = ri.nonRelFockMatrix(hs, src, D)
    assert np.abs(F - ro.nonrel_fock(hs, B, D, Ss, Xs)).max() < 1e-10
