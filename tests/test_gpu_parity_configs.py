"""Parity at the full sizes the bench measures, against the reference compiled from its own sources
(oracle/_ref), on the bench's own inputs:

* the nonrelativistic RI Fock build at n = 400, naux = 1600, nocc = 40 (nonRelFockMatrix,
  src/NON_REL/NonRelFockMatrixRi.cpp:27-100): the 40 x 80 half-transform tiles, the split-K SYRK and
  the recovery's early exit all run at this shape only;
* the 4-component RKB Fock build at nl = 200, ns = 600, naux = 1000, 20 Kramers pairs (rkbFockMatrix,
  src/UKB/UkbFockMatrixRi.cpp:185-216): 80 x 80 batched tiles for the 80-row [Re; Im] blocks, Gauss's
  three-product blocks and the sixteen-wave split rule;
* the largest instance of the X2C geometry scan, nl = 120, naux = 480 (x2cFockMatrix,
  src/X2C_DHF/X2C_FockMatrixRi.cpp:35-162, and the SCF loop, src/X2C_DHF/X2C_HF.cpp:43-138);
* the X2C-HF time-to-convergence system (400 spinors, naux 1000): FP64 and mixed loops against the
  reference's FP64 loop.

Bar: max |F_gpu - F_ref| <= 1e-10 (FP64) and converged energies within 1e-8 Ha."""
import os

import numpy as np
import pytest

import bench
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import ri, scf  # noqa: E402

TOL = 1e-10


@pytest.fixture(scope="module")
def ref_all(ref_lib):
    ref_lib.set_threads(os.cpu_count() or 1)
    yield ref_lib
    ref_lib.set_threads(4)


def test_nonrel_fock_headline_shape(ref_all):
    inp = bench.make_inputs()
    src = ri.RiNonRelEriSource(bench.N_AO, inp["B"], inp["X"], inp["S"])
    F = ri.nonRelFockMatrix(inp["h"], src, inp["D"])
    Fr = ref_all.nonrel_fock(inp["h"], inp["B"], inp["D"], inp["S"], inp["X"])
    err = np.abs(F - Fr).max()
    print(f"n=400 naux=1600 nocc=40: max|F - F_ref| = {err:.3e}")
    assert err <= TOL
    src.store.close()


def test_rkb_fock_4c_shape(ref_all):
    s = synth.rkb_system(bench.NL4, bench.NS4, bench.NAUX4, 2 * (bench.NOCC4 // 2), seed=bench.SEED + 11, box=20.0)
    src = ri.RiDirectEriSource(bench.NL4, bench.NS4, s["B_LL"], s["B_SS"], s["v_total"], s["s_full"], s["x_full"])
    F = ri.rkbFockMatrix(s["h"], src, s["P0"])
    Fr = ref_all.rkb_fock(s["h"], bench.NL4, bench.NS4, s["B_LL"], s["B_SS"], s["v_total"], s["s_full"],
                          s["x_full"], s["P0"])
    err = np.abs(F - Fr).max()
    print(f"nl=200 ns=600 naux=1000 40 spinors: max|F - F_ref| = {err:.3e}")
    assert err <= TOL
    src.store.close()


def test_x2c_scan_largest_instance(ref_all):
    s = synth.x2c_system(120, 480, 14, seed=bench.SEED + 100)
    src = ri.RiX2cEriSource(120, s["B"], s["X"], s["S"])
    F = ri.x2cFockMatrix(s["h"], src, s["P0"])
    Fr = ref_all.x2c_fock(s["h"], s["B"], s["P0"], s["S"], s["X"])
    assert np.abs(F - Fr).max() <= TOL
    r = scf.runX2CHartreeFockScf(s["h"], src, s["X"], s["P0"], 14)
    rr = ref_all.x2c_scf(s)
    assert r["converged"] and rr["converged"]
    assert r["iterations"] == rr["iterations"]
    assert np.abs(r["history"] - rr["history"]).max() <= 1e-8
    rm = scf.runX2CHartreeFockScf(s["h"], src, s["X"], s["P0"], 14, precision="mixed")
    assert rm["converged"] and abs(rm["energy"] - rr["energy"]) <= 1e-8
    src.store.close()


def test_x2c_time_to_convergence_system(ref_all):
    s = synth.x2c_system(bench.X2C_NL, bench.X2C_NAUX, bench.X2C_NE, seed=bench.SEED + 21, box=20.0, gap=bench.X2C_GAP)
    s["B"] = s["B"] * bench.X2C_B
    src = ri.RiX2cEriSource(bench.X2C_NL, s["B"], s["X"], s["S"])
    rr = ref_all.x2c_scf(s)
    assert rr["converged"]
    for prec in ("fp64", "mixed"):
        r = scf.runX2CHartreeFockScf(s["h"], src, s["X"], s["P0"], bench.X2C_NE, precision=prec)
        print(f"X2C-HF 400 spinors {prec}: E - E_ref = {r['energy'] - rr['energy']:.3e} Ha")
        assert r["converged"] and abs(r["energy"] - rr["energy"]) <= 1e-8
    src.store.close()
