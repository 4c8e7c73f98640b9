"""Device-resident SCF loops against the reference's own loops (golden histories from the compiled
reference and the numpy restatement): energies per iteration to 1e-8 Ha, same iteration count;
mixed precision converges to the FP64 energy within 1e-8 Ha."""
import numpy as np
import pytest

from conftest import golden
from oracle import ri_oracle as o
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import ri, scf  # noqa: E402


def _run(sysd, **kw):
    src = ri.RiNonRelEriSource(sysd["h"].shape[0], sysd["B"], sysd["X"], sysd["S"])
    return scf.runNonRelativisticHartreeFock(src, sysd["h"], sysd["X"], sysd["D0"], int(sysd["n_electrons"]), **kw)


def test_nonrel_golden_history():
    g = golden("scf_nonrel")
    r = _run(g)
    assert r["converged"]
    assert r["iterations"] == int(g["iterations"])
    assert np.abs(r["history"] - g["history"]).max() <= 1e-8
    assert np.abs(r["P"] - g["P"]).max() <= 1e-6


@pytest.mark.parametrize("n,naux,nocc,seed", [(24, 129, 5, 1), (60, 200, 8, 2), (100, 300, 12, 3)])
def test_nonrel_vs_oracle(n, naux, nocc, seed):
    s = synth.nonrel_system(n, naux, nocc, seed=seed)
    r = _run(s)
    ro = o.nonrel_scf(s)
    assert r["converged"] and ro["converged"]
    assert abs(r["energy"] - ro["energy"]) <= 1e-8
    assert r["iterations"] == ro["iterations"]


@pytest.mark.parametrize("n,naux,nocc,seed", [(60, 200, 8, 4), (128, 400, 16, 5)])
def test_nonrel_mixed_reaches_fp64_energy(ref_lib, n, naux, nocc, seed):
    s = synth.nonrel_system(n, naux, nocc, seed=seed)
    r64 = _run(s)
    rr = ref_lib.nonrel_scf(s)  # the reference's own FP64 loop
    assert rr["converged"] and abs(r64["energy"] - rr["energy"]) <= 1e-8
    for switch in (0.0, 1e-5):  # incremental only / one FP64 re-seed of the accumulated exchange
        rm = _run(s, precision="mixed", mixed_switch=switch)
        assert r64["converged"] and rm["converged"]
        assert rm["mixed_iterations"] >= 1
        # the first build, the optional re-seed and the final build are the FP64 ones
        assert rm["fp64_iterations"] == (2 if switch == 0.0 else rm["fp64_iterations"]) <= 3
        assert rm["iterations"] == rm["mixed_iterations"] + rm["fp64_iterations"]
        assert abs(rm["energy"] - r64["energy"]) <= 1e-8
        assert abs(rm["energy"] - rr["energy"]) <= 1e-8


def _run_x2c(sysd, **kw):
    src = ri.RiX2cEriSource(int(sysd["h"].shape[0]) // 2, sysd["B"], sysd["X"], sysd["S"])
    return scf.runX2CHartreeFockScf(sysd["h"], src, sysd["X"], sysd["P0"], int(sysd["n_electrons"]), **kw)


def _run_dhf(sysd, **kw):
    src = ri.RiDirectEriSource(int(sysd["nl"]), int(sysd["ns"]), sysd["B_LL"], sysd["B_SS"], sysd["v_total"],
                               sysd["s_full"], sysd["x_full"])
    return scf.runDiracHartreeFockScf(sysd["h"], src, sysd["x_full"], sysd["P0"], int(sysd["n_electrons"]), **kw)


def test_x2c_golden_history():
    g = golden("scf_x2c")
    r = _run_x2c(g)
    assert r["converged"]
    assert r["iterations"] == int(g["iterations"])
    assert np.abs(r["history"] - g["history"]).max() <= 1e-8
    assert np.abs(r["P"] - g["P"]).max() <= 1e-6


def test_dhf_golden_history():
    g = golden("scf_dhf")
    r = _run_dhf(g)
    assert r["converged"]
    assert r["iterations"] == int(g["iterations"])
    assert np.abs(r["history"] - g["history"]).max() <= 1e-8
    assert np.abs(r["P"] - g["P"]).max() <= 1e-6


@pytest.mark.parametrize("nl,naux,ne,seed", [(12, 60, 6, 21), (40, 160, 10, 22)])
def test_x2c_vs_reference(ref_lib, nl, naux, ne, seed):
    s = synth.x2c_system(nl, naux, ne, seed=seed)
    r = _run_x2c(s)
    rr = ref_lib.x2c_scf(s)
    assert r["converged"] and rr["converged"]
    assert r["iterations"] == rr["iterations"]
    assert np.abs(r["history"] - rr["history"]).max() <= 1e-8


@pytest.mark.parametrize("nl,ns,naux,ne,seed", [(6, 11, 40, 4, 23), (12, 25, 80, 8, 24)])
def test_dhf_vs_reference(ref_lib, nl, ns, naux, ne, seed):
    s = synth.rkb_system(nl, ns, naux, ne, seed=seed)
    r = _run_dhf(s)
    rr = ref_lib.dhf_scf(s)
    assert r["converged"] and rr["converged"]
    assert r["iterations"] == rr["iterations"]
    assert np.abs(r["history"] - rr["history"]).max() <= 1e-8


def test_x2c_without_kramers_projection_and_with_mixing(ref_lib):
    s = synth.x2c_system(10, 50, 6, seed=25)
    r = _run_x2c(s, kramers_restricted=False)
    rr = ref_lib.x2c_scf(s, kramers=False)
    assert r["iterations"] == rr["iterations"]
    assert np.abs(r["history"] - rr["history"]).max() <= 1e-8
    # plain linear mixing (no DIIS) reaches the same state; tight tolerances because the reference's
    # OR rule stops a slowly mixed iteration as soon as one step changes E by less than tolE
    rm = _run_x2c(s, diis_size=0, mixing=0.5, max_iterations=400, energy_tolerance=1e-13, density_tolerance=1e-10)
    assert rm["converged"] and abs(rm["energy"] - r["energy"]) <= 1e-7


def test_x2c_batch_matches_single_runs(ref_lib):
    systems = [synth.x2c_system(nl, 4 * nl, ne, seed=30 + k) for k, (nl, ne) in
               enumerate([(8, 4), (14, 6), (20, 4), (11, 2), (17, 8), (9, 4)])]
    probs = []
    for s in systems:
        src = ri.RiX2cEriSource(s["nl"], s["B"], s["X"], s["S"])
        probs.append(dict(eri=src, h_x2c=s["h"], x_large=s["X"], initial_density=s["P0"], n_electrons=s["n_electrons"]))
    batch = scf.runX2CHartreeFockScfBatch(probs, workers=3)
    for s, b in zip(systems, batch):
        single = _run_x2c(s)
        assert b["converged"] and b["iterations"] == single["iterations"]
        assert np.array_equal(b["history"], single["history"])
    rr = ref_lib.x2c_scf(systems[2])
    assert np.abs(batch[2]["history"] - rr["history"]).max() <= 1e-8
