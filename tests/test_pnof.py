"""PNOF / GNOF functionals (rerdmft_b200.pnof) against the reference compiled from its sources: the
actual-orbital two-RDM factors (buildPnofFullTwoRdm, PnofFock.cpp:29), the energy and its occupation
gradient (pnofElectronicEnergy / pnofOccupationGradient, PNOFs.cpp:271, :463), and the occupation step
at fixed orbitals."""
import numpy as np
import pytest

from oracle import ri_oracle as o
from rerdmft_b200 import pnof, synth


def _setup(n, nocc, coupling, n_sub, seed):
    f = synth.functional_system(n, 24, seed, nocc=nocc)
    gem = pnof.nonrel_geminals(n, nocc, coupling, n_sub)
    H = np.zeros((2 * n, 2 * n))
    H[:n, :n] = f["h"]
    H[n:, n:] = f["h"]
    J, K, _ = o.jkl_matrices(o.nonrel_mo_embedded(f["Bmo"], n), 2 * n)
    return f, gem, H, J, K


@pytest.mark.parametrize("functional", ["PNOF5", "PNOF7", "PNOF7S", "GNOF"])
@pytest.mark.parametrize("n,nocc,coupling,n_sub", [(8, 2, 3, 2), (9, 3, 3, 2), (10, 2, 4, 1)])
def test_two_rdm_and_energy_match_reference(ref_lib, functional, n, nocc, coupling, n_sub):
    f, gem, H, J, K = _setup(n, nocc, coupling, n_sub, seed=n + nocc)
    rng = np.random.default_rng(n)
    occ = pnof.occupations_of(gem, coupling, rng.uniform(0.1, 1.4, size=n_sub * (coupling - 1)), 2 * n)
    fid = pnof.FUNCTIONALS[functional]
    mine = pnof.full_two_rdm(fid, gem, occ, 2 * n)
    ref = ref_lib.pnof_full_two_rdm(functional, gem, occ, 2 * n, relativistic=False)
    for k in ("two_rdm_h", "two_rdm_x", "two_rdm_l1", "two_rdm_l2"):
        assert np.abs(mine[k] - ref[k]).max() <= 1e-15, k
    assert np.array_equal(mine["pair_of"], ref["pair_of"])
    e_ref, g_ref = ref_lib.pnof_energy_nonrel(functional, gem, occ, f["Bmo"], n, H)
    e = pnof.electronic_energy(fid, gem, occ, np.diag(H), J, K)
    assert abs(e - e_ref) <= 1e-12 * max(1.0, abs(e_ref))
    # the occupation gradient per geminal (both members of a geminal move together)
    for a, g in enumerate(gem):
        if g[3] and (gem[:, 2] == g[2]).sum() == 1:
            continue  # frozen pair: n = 1 sits on the edge of GNOF's square roots
        d = np.zeros(2 * n)
        d[g[0]] = d[g[1]] = 1e-6
        fd = (pnof.electronic_energy(fid, gem, occ + d, np.diag(H), J, K) -
              pnof.electronic_energy(fid, gem, occ - d, np.diag(H), J, K)) / 2e-6
        assert abs(fd - g_ref[a]) <= 1e-6 * max(1.0, abs(g_ref[a])), (a, fd, g_ref[a])


def test_occupation_step_reaches_a_stationary_point(ref_lib):
    n, nocc, coupling = 8, 2, 3
    f, gem, H, J, K = _setup(n, nocc, coupling, 2, seed=4)
    fid = pnof.FUNCTIONALS["GNOF"]
    g0 = np.full(2 * (coupling - 1), np.pi / 4)
    r = pnof.optimize_occupations(fid, gem, coupling, np.diag(H), J, K, g0, 2 * n)
    assert r["converged"]
    e0 = pnof.electronic_energy(fid, gem, pnof.occupations_of(gem, coupling, g0, 2 * n), np.diag(H), J, K)
    assert r["energy"] < e0
    e_ref, g_ref = ref_lib.pnof_energy_nonrel("GNOF", gem, r["occupations"], f["Bmo"], n, H)
    assert abs(r["energy"] - e_ref) <= 1e-12 * max(1.0, abs(e_ref))
    # stationary in the angles: the reference gradient contracted with d occ / d gamma vanishes
    for k in range(r["gammas"].size):
        d = np.zeros_like(r["gammas"])
        d[k] = 1e-6
        dn = (pnof.occupations_of(gem, coupling, r["gammas"] + d, 2 * n) -
              pnof.occupations_of(gem, coupling, r["gammas"] - d, 2 * n)) / 2e-6
        dg = sum(g_ref[a] * dn[g[0]] for a, g in enumerate(gem))
        assert abs(dg) <= 1e-6, (k, dg)
