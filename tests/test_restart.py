"""RESTART files: the library's writer and reader against the reference's own writeRestart / readRestart
(src/Utils/Restart.cpp, compiled from its sources), byte for byte, for every kind; the reference's
error checks.  Host code only (no GPU)."""
import ctypes

import numpy as np
import pytest

from rerdmft_b200 import _lib as L
from rerdmft_b200.restart import RestartData, readRestart, writeRestart


def _cases():
    rng = np.random.default_rng(5)
    yield RestartData("NON_REL", "GNOF", "GAMMAS", 0x1234ABCD5678EF01, 4, 2, 3, 1, 0, 0, -7.9976533572, True, True,
                      rng.random(22), rng.standard_normal(4), np.zeros(0), rng.standard_normal((22, 22)))
    yield RestartData("X2C", "MULLER", "OCCUPATIONS", 42, 4, 0, 0, 0, 1, 5, -7.99846, False, True, rng.random(22),
                      np.zeros(0), np.zeros(0), rng.standard_normal((22, 22)) + 1j * rng.standard_normal((22, 22)))
    yield RestartData("4C", "PCCD", "PCCD", 7, 4, 0, 0, 0, 1, 2, -7.99841, True, False, rng.random(44), np.zeros(0),
                      rng.standard_normal(12), rng.standard_normal((44, 44)) + 1j * rng.standard_normal((44, 44)))
    yield RestartData("X2C", "CASSCF", "CASSCF", 9, 4, 0, 0, 0, 0, 0, -7.9801, True, True, rng.random(10), np.zeros(0),
                      np.zeros(0), rng.standard_normal((10, 10)) + 1j * rng.standard_normal((10, 10)), 2, 4,
                      rng.standard_normal(12))


def _fields(d, keep):
    """rr_restart record of RestartData d (arrays kept alive in keep)."""
    def vec(a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        keep.append(a)
        return (a.ctypes.data if a.size else None), a.size
    C = np.ascontiguousarray(d.coefficients)
    keep.append(C)
    o, g, a, c = vec(d.occupations), vec(d.gammas), vec(d.amplitudes), vec(d.cas_state)
    return L.Restart(d.method.encode(), d.functional.encode(), d.kind.encode(), d.basis_fingerprint, d.n_electrons,
                     d.pnof_subspaces, d.pnof_coupling, d.n_core, d.jk_frozen_pairs, d.jk_active_pairs,
                     d.total_energy, int(d.orbitals_optimized), int(d.converged), o[0], o[1], g[0], g[1], a[0], a[1],
                     int(np.iscomplexobj(C)), C.shape[0], C.shape[1], C.ctypes.data, d.cas_electrons, d.cas_spinors,
                     c[0], c[1])


def _same(a: RestartData, b: RestartData):
    for k in ("method", "functional", "kind", "basis_fingerprint", "n_electrons", "pnof_subspaces", "pnof_coupling",
              "n_core", "jk_frozen_pairs", "jk_active_pairs", "total_energy", "orbitals_optimized", "converged",
              "cas_electrons", "cas_spinors"):
        assert getattr(a, k) == getattr(b, k), k
    for k in ("occupations", "gammas", "amplitudes", "cas_state", "coefficients"):
        assert np.array_equal(np.asarray(getattr(a, k)), np.asarray(getattr(b, k))), k


@pytest.mark.parametrize("case", list(range(4)))
def test_byte_identical_both_ways(ref_lib, tmp_path, case):
    d = list(_cases())[case]
    ours, theirs, back = tmp_path / "ours.bin", tmp_path / "theirs.bin", tmp_path / "back.bin"
    writeRestart(ours, d)
    keep = []
    ref_lib.restart_write(theirs, _fields(d, keep))
    assert ours.read_bytes() == theirs.read_bytes()
    ref_lib.restart_rewrite(ours, back)  # the reference reads our file and writes the same bytes
    assert back.read_bytes() == ours.read_bytes()
    _same(readRestart(theirs), d)


def test_version_2_files_are_read(ref_lib, tmp_path):
    d = list(_cases())[0]
    p3, p2 = tmp_path / "v3.bin", tmp_path / "v2.bin"
    writeRestart(p3, d)
    raw = bytearray(p3.read_bytes())
    raw[8:12] = (2).to_bytes(4, "little")
    p2.write_bytes(bytes(raw[: len(raw) - 24]))  # no CASSCF section: two int64 and an empty vector
    r = readRestart(p2)
    _same(r, d)
    ref_lib.restart_rewrite(p2, tmp_path / "v2_back.bin")  # the reference reads it too (and writes version 3)
    assert (tmp_path / "v2_back.bin").read_bytes() == p3.read_bytes()


def test_errors_like_reference(tmp_path):
    d = list(_cases())[0]
    bad = RestartData(**{**d.__dict__, "kind": "NOPE"})
    with pytest.raises(L.RrError, match="kind must be OCCUPATIONS, GAMMAS, PCCD or CASSCF"):
        writeRestart(tmp_path / "x.bin", bad)
    with pytest.raises(L.RrError, match="kind GAMMAS without gamma angles"):
        writeRestart(tmp_path / "x.bin", RestartData(**{**d.__dict__, "gammas": np.zeros(0)}))
    with pytest.raises(L.RrError, match="coefficient matrix is missing"):
        writeRestart(tmp_path / "x.bin", RestartData(**{**d.__dict__, "coefficients": np.zeros((0, 0))}))
    p = tmp_path / "t.bin"
    writeRestart(p, d)
    p.write_bytes(p.read_bytes()[:100])
    with pytest.raises(L.RrError, match="truncated"):
        readRestart(p)
    (tmp_path / "m.bin").write_bytes(b"NOTRERDM" + bytes(64))
    with pytest.raises(L.RrError, match="is not a RERDMFT restart file"):
        readRestart(tmp_path / "m.bin")
