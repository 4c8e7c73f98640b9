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
def test_nonrel_mixed_reaches_fp64_energy(n, naux, nocc, seed):
    s = synth.nonrel_system(n, naux, nocc, seed=seed)
    r64 = _run(s)
    rm = _run(s, precision="mixed", mixed_switch=1e-5)
    assert r64["converged"] and rm["converged"]
    assert rm["mixed_iterations"] >= 1 and rm["fp64_iterations"] >= 1
    assert abs(rm["energy"] - r64["energy"]) <= 1e-8
