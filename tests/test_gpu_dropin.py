"""The C++ drop-in (include/rr_ri.hpp) inside the reference's own code.

oracle/_ref/librrref_dropin.so is the reference's SCF loops, DIIS, linear algebra and bridge,
compiled from its sources, with its six RI .cpp files replaced by rr_ri.hpp over librr_ri.  Every
golden case made from the pure reference is replayed through it: the reference's call sites, now
running the GPU path, must give the reference's answers (the SCF loops iteration by iteration).
Runs in a child process so that the two builds of the reference never share one process."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
TOL = 1e-10


def _cases():
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import GOLDEN, golden
    from oracle import ref

    assert ref.LIB_PATH == ref.DROPIN_PATH
    ref.set_threads(2)
    for p in sorted(GOLDEN.glob("nonrel_fock_*.npz")):
        g = golden(p.stem)
        for _ in range(2):  # the second call reuses the resident tensor
            assert np.abs(ref.nonrel_fock(g["h"], g["B"], g["D"], g["S"], g["X"]) - g["F"]).max() <= TOL, p.stem
        if "D_mix" in g:
            assert np.abs(ref.nonrel_fock(g["h"], g["B"], g["D_mix"], g["S"], g["X"]) - g["F_mix"]).max() <= TOL
    # B rewritten in the same host buffer (one symmetric pair of entries of one aux row changed): the
    # resident-tensor cache must see the new contents and upload them
    from oracle import ri_oracle
    g = golden("nonrel_fock_n24_naux129")
    B2 = g["B"].copy()
    B2[77, 5 * 24 + 17] += 0.25
    B2[77, 17 * 24 + 5] += 0.25
    F2 = ref.nonrel_fock(g["h"], B2, g["D"], g["S"], g["X"])
    assert np.abs(F2 - ri_oracle.nonrel_fock(g["h"], B2, g["D"], g["S"], g["X"])).max() <= TOL
    assert np.abs(F2 - g["F"]).max() > 1e-6
    for p in sorted(GOLDEN.glob("x2c_fock_*.npz")):
        g = golden(p.stem)
        assert np.abs(ref.x2c_fock(g["h"], g["B"], g["P"], g["S"], g["X"]) - g["F"]).max() <= TOL, p.stem
    for p in sorted(GOLDEN.glob("rkb_fock_*.npz")):
        g = golden(p.stem)
        nl, ns = int(round(g["B_LL"].shape[1] ** 0.5)), int(round(g["B_SS"].shape[1] ** 0.5))
        F = ref.rkb_fock(g["h"], nl, ns, g["B_LL"], g["B_SS"], g["v_total"], g["s_full"], g["x_full"], g["P"])
        assert np.abs(F - g["F"]).max() <= TOL, p.stem
        G = ref.ukb_two_electron(nl, ns, g["B_LL"], g["B_SS"], g["P_ukb"], g["C_occ"], g["occ"])
        assert np.abs(G - g["G"]).max() <= TOL, p.stem

    g = golden("nonrel_mo")
    n = g["C"].shape[0]
    assert np.abs(ref.nonrel_mo_build(g["B"], g["C"]) - g["Bmo"]).max() <= TOL
    assert np.abs(ref.nonrel_mo_rotated(g["Bmo"], n, g["U"]) - g["Brot"]).max() <= TOL
    g = golden("ri_mo")
    nl, ns = int(round(g["B_LL"].shape[1] ** 0.5)), int(round(g["B_SS"].shape[1] ** 0.5))
    nt = g["c_ukb"].shape[1]
    assert np.abs(ref.ri_mo_build(nl, ns, g["B_LL"], g["B_SS"], g["c_ukb"]) - g["Bmo"]).max() <= TOL
    assert np.abs(ref.ri_mo_rotated(g["Bmo"], nt, g["U"]) - g["Brot"]).max() <= TOL
    assert np.abs(ref.ri_mo_positive(g["Bmo"], nt, 4) - g["Bpos"]).max() == 0.0
    g = golden("hx_fock")
    Fc = ref.hx_fock_complex(g["Bc"], g["hc"].shape[0], g["hc"], g["occ"], g["h2"], g["x2"], g["po"], g["l1"], g["l2"])
    assert np.abs(Fc - g["Fc"]).max() <= TOL
    nsp = int(round(g["Bmo"].shape[1] ** 0.5))
    Fr = ref.hx_fock_nonrel(g["Bmo"], nsp, g["hr"], g["occr"], g["h2r"], g["x2r"], g["por"], g["l1r"], g["l2r"])
    assert np.abs(Fr - g["Fr"]).max() <= TOL

    g = golden("scf_nonrel")
    r = ref.nonrel_scf(dict(n=g["h"].shape[0], B=g["B"], h=g["h"], S=g["S"], X=g["X"], D0=g["D0"],
                            n_electrons=int(g["n_electrons"])))
    assert r["iterations"] == int(g["iterations"]) and np.abs(r["history"] - g["history"]).max() <= 1e-9
    g = golden("scf_x2c")
    r = ref.x2c_scf(dict(nl=g["h"].shape[0] // 2, B=g["B"], h=g["h"], S=g["S"], X=g["X"], P0=g["P0"],
                         n_electrons=int(g["n_electrons"])))
    assert r["iterations"] == int(g["iterations"]) and np.abs(r["history"] - g["history"]).max() <= 1e-9
    g = golden("scf_dhf")
    sysd = {k: g[k] for k in ("B_LL", "B_SS", "v_total", "s_full", "x_full", "h", "P0")}
    sysd.update(nl=int(g["nl"]), ns=int(g["ns"]), n_rkb=g["h"].shape[0], n_electrons=int(g["n_electrons"]))
    r = ref.dhf_scf(sysd)
    assert r["iterations"] == int(g["iterations"]) and np.abs(r["history"] - g["history"]).max() <= 1e-9
    print("DROPIN-OK")


def test_reference_call_sites_on_the_gpu_path():
    lib = ROOT / "oracle" / "_ref" / "librrref_dropin.so"
    if not lib.exists():
        pytest.skip("oracle/_ref/librrref_dropin.so not built (make -C oracle dropin needs the reference tree)")
    env = dict(os.environ, RRREF_LIB="dropin")
    p = subprocess.run([sys.executable, __file__], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and "DROPIN-OK" in p.stdout, p.stdout[-3000:] + p.stderr[-3000:]


if __name__ == "__main__":
    _cases()
