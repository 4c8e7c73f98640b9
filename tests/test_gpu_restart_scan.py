"""The hand-over between the runs of a geometry scan through RESTART files: the converged X2C-HF orbitals
of one geometry (the loop's c_matrix) are written with the library's writer, read back, rotated
(restartCoefficients, src/Utils/Restart.cpp:199-206, on the GPU) and turned into the next geometry's
starting density on the GPU.  The next run converges in fewer iterations than from the core guess, to the
energy of the reference's own loop started from the same density (compiled from its sources)."""
import numpy as np
import pytest

from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import ri, scf  # noqa: E402
from rerdmft_b200.restart import RestartData, densityFromOrbitals, readRestart, restartCoefficients, writeRestart  # noqa: E402


def test_restart_coefficients_and_density():
    rng = np.random.default_rng(3)
    C = rng.standard_normal((30, 20)) + 1j * rng.standard_normal((30, 20))
    U = rng.standard_normal((20, 20)) + 1j * rng.standard_normal((20, 20))
    assert np.abs(restartCoefficients(C, U) - C @ U).max() <= 1e-12
    assert np.array_equal(restartCoefficients(C), C)
    occ = np.r_[np.ones(6), np.zeros(14)]
    P = densityFromOrbitals(C, occ)
    assert np.abs(P - (C * occ) @ C.conj().T).max() <= 1e-12
    Cr = rng.standard_normal((25, 25))
    assert np.abs(densityFromOrbitals(Cr, 2.0 * np.r_[np.ones(4), np.zeros(21)]) - 2.0 * Cr[:, :4] @ Cr[:, :4].T).max() <= 1e-12


def test_scan_step_through_restart(ref_lib, tmp_path):
    nl, naux, ne = 40, 160, 10
    a = synth.x2c_system(nl, naux, ne, seed=22)
    ra = scf.runX2CHartreeFockScf(a["h"], ri.RiX2cEriSource(nl, a["B"], a["X"], a["S"]), a["X"], a["P0"], ne,
                                  orbitals=True)
    assert ra["converged"]
    occ = np.r_[np.ones(ne), np.zeros(ra["c_matrix"].shape[1] - ne)]
    writeRestart(tmp_path / "RESTART.X2C", RestartData("X2C", "HF", "OCCUPATIONS", 1, ne, total_energy=ra["energy"],
                                                        converged=True, occupations=occ,
                                                        coefficients=ra["c_matrix"]))
    rd = readRestart(tmp_path / "RESTART.X2C")
    C = restartCoefficients(rd.coefficients)  # no orbital optimisation: the identity rotation
    P_next = densityFromOrbitals(C, rd.occupations)
    # the next geometry of the scan: the same system with its three-centre tensor scaled by 1 %
    b = dict(a)
    b["B"] = a["B"] * 1.01
    src_b = ri.RiX2cEriSource(nl, b["B"], b["X"], b["S"])
    cold = scf.runX2CHartreeFockScf(b["h"], src_b, b["X"], b["P0"], ne)
    warm = scf.runX2CHartreeFockScf(b["h"], src_b, b["X"], P_next, ne)
    assert cold["converged"] and warm["converged"]
    assert warm["iterations"] < cold["iterations"]
    rr = ref_lib.x2c_scf(dict(b, P0=P_next))
    assert rr["converged"] and warm["iterations"] == rr["iterations"]
    assert np.abs(warm["history"] - rr["history"]).max() <= 1e-8
