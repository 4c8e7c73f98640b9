"""Writes the molecular fixtures of the integral engine from the reference's own example data.

For each molecule: the basis set file the reference's example names (parsed by
``rerdmft_b200.basis.read_basis_set``, stored per element as shells), the geometry (converted to bohr
as the reference's input reader does) and the total RI Hartree-Fock energy the reference printed for
that input (``examples/reference.yaml``, "Total nonrelativistic HF energy#1").  The energies were
computed by the reference with libcint's integrals; these fixtures let the tests pin this repository's
integrals end to end without the reference tree.

    REF_ROOT=<reference checkout> python tests/golden/make_integrals_golden.py

Molecules: LiH / 6-31G at 1.5949 Angstrom (lih_gnof_full_optimization_use_ri_nonrel_x2c.inp, USE_RI TRUE,
the dense-integral value of the same geometry alongside from lih_gnof_full_optimization.inp) and at
5.0 Angstrom (casscf_lih_dissociated_core.inp, RI by default); the water / cc-pVDZ and CO / cc-pVDZ basis
sets (d functions) for device-against-oracle parity without a reference energy.
"""
from __future__ import annotations

import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from rerdmft_b200 import basis as bs  # noqa: E402

OUT = Path(__file__).resolve().parent
REF = Path(os.environ.get("REF_ROOT", "/root/reference"))


def yaml_energy(key: str, label: str) -> float:
    """The value of `label` in the block `key:` of examples/reference.yaml (a plain text scan)."""
    text = (REF / "examples" / "reference.yaml").read_text().splitlines()
    inside = False
    for line in text:
        if re.match(rf"^{re.escape(key)}:\s*$", line):
            inside = True
            continue
        if inside and re.match(r"^\S", line):
            break
        if inside and line.strip().startswith(label + ":"):
            return float(line.split(":", 1)[1])
    raise KeyError(f"{key} / {label}")


def geometry_of(inp: str) -> tuple[list, int]:
    lines = (REF / "examples" / inp).read_text().splitlines()
    nelec = None
    geo = []
    inside = False
    for raw in lines:
        line = raw.split("#")[0].split("!")[0].strip()
        if not line:
            continue
        up = line.upper()
        if up.startswith("NELEC"):
            nelec = int(line.split()[1])
        elif up == "GEOMETRY":
            inside = True
        elif up == "END":
            inside = False
        elif inside:
            s, x, y, z = line.split()[:4]
            geo.append((s, float(x) * bs.ANGSTROM_TO_BOHR, float(y) * bs.ANGSTROM_TO_BOHR,
                        float(z) * bs.ANGSTROM_TO_BOHR))
    return geo, nelec


def basis_arrays(path: Path) -> dict:
    sets = bs.read_basis_set(str(path))
    el, ls, npr, ex, co = [], [], [], [], []
    for e, shells in sets.items():
        for sh in shells:
            el.append(e)
            ls.append(sh.l)
            npr.append(len(sh.exponents))
            ex.extend(sh.exponents)
            co.extend(sh.coefficients)
    return dict(shell_element=np.array(el), shell_l=np.array(ls, dtype=np.int32),
                shell_nprim=np.array(npr, dtype=np.int32), exponents=np.array(ex), coefficients=np.array(co))


def save_molecule(name, gbs, inp=None, geometry=None, nelec=None, energies=None):
    arrays = basis_arrays(REF / "examples" / gbs)
    if inp:
        geometry, nelec = geometry_of(inp)
    arrays["atom_symbol"] = np.array([g[0] for g in geometry])
    arrays["atom_xyz"] = np.array([g[1:] for g in geometry], dtype=np.float64)
    arrays["nelec"] = np.array(nelec)
    for k, v in (energies or {}).items():
        arrays[k] = np.array(v)
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    print(f"  {name}.npz")


def main():
    save_molecule("lih_631g", "lih-6-31g.gbs", inp="lih_gnof_full_optimization_use_ri_nonrel_x2c.inp",
                  energies=dict(
                      e_hf_ri=yaml_energy("lih_gnof_full_optimization_use_ri_nonrel_x2c",
                                          "Total nonrelativistic HF energy#1"),
                      e_hf_dense=yaml_energy("lih_gnof_full_optimization", "Total nonrelativistic HF energy#1"),
                      tolerance=1e-6))
    save_molecule("lih_631g_5a", "lih-6-31g.gbs", inp="casscf_lih_dissociated_core.inp",
                  energies=dict(e_hf_ri=yaml_energy("casscf_lih_dissociated_core", "Total nonrelativistic HF energy#1"),
                                tolerance=1e-6))
    save_molecule("water_ccpvdz", "water-cc-pvdz.gbs", inp="water.inp")
    save_molecule("co_ccpvdz", "co-cc-pvdz.gbs", inp="co-cc-pvdz.inp")


if __name__ == "__main__":
    main()
