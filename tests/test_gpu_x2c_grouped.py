"""The lockstep X2C-HF batch (rr_scf_run_x2c_grouped: every phase of an iteration one grouped launch for
all instances) against the reference's own SCF loop (X2C_HF.cpp:43-138, compiled oracle) per instance,
against the single-instance device loop, and against itself run one instance at a time (bit for bit);
its launch count per iteration does not grow with the number of instances; the autotuner cache file
round-trips."""
import numpy as np
import pytest

from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import ri, scf  # noqa: E402

SHAPES = [(20, 4), (33, 14), (48, 4), (26, 14), (60, 4), (41, 14)]


def _systems(shapes, seed0=300):
    return [synth.x2c_system(nl, 4 * nl, ne, seed=seed0 + k) for k, (nl, ne) in enumerate(shapes)]


def _problems(systems):
    out = []
    for s in systems:
        src = ri.RiX2cEriSource(s["nl"], s["B"], s["X"], s["S"])
        out.append(dict(eri=src, h_x2c=s["h"], x_large=s["X"], initial_density=s["P0"],
                        n_electrons=s["n_electrons"]))
    return out


def _close(probs):
    for p in probs:
        p["eri"].store.close()


def test_grouped_batch_matches_reference_and_single_runs(ref_lib):
    systems = _systems(SHAPES)
    probs = _problems(systems)
    st = {}
    batch = scf.runX2CHartreeFockScfBatch(probs, mode="grouped", stats=st)
    assert st["grouped_instances_first"] == len(SHAPES)
    for k, (s, b) in enumerate(zip(systems, batch)):
        rr = ref_lib.x2c_scf(s)
        assert b["converged"] and rr["converged"]
        assert b["iterations"] == rr["iterations"], k
        assert np.abs(b["history"] - rr["history"]).max() <= 1e-8, k
        single = scf.runX2CHartreeFockScf(s["h"], probs[k]["eri"], s["X"], s["P0"], s["n_electrons"])
        assert abs(b["energy"] - single["energy"]) <= 1e-9
        assert np.abs(b["P"] - single["P"]).max() <= 1e-7
    _close(probs)


def test_grouped_results_do_not_depend_on_the_batch():
    systems = _systems(SHAPES[:4], seed0=320)
    probs = _problems(systems)
    batch = scf.runX2CHartreeFockScfBatch(probs, mode="grouped")
    for k in range(len(probs)):
        alone = scf.runX2CHartreeFockScfBatch([probs[k]], mode="grouped")[0]
        assert alone["iterations"] == batch[k]["iterations"]
        assert np.array_equal(alone["history"], batch[k]["history"])
        assert np.array_equal(alone["P"], batch[k]["P"])
    _close(probs)


def test_launches_per_iteration_do_not_grow_with_the_batch():
    systems = _systems(SHAPES[:3], seed0=340)
    small = _problems(systems)
    big = _problems(systems + systems + systems)
    s1, s3 = {}, {}
    scf.runX2CHartreeFockScfBatch(small, mode="grouped", stats=s1)  # tunes every shape
    scf.runX2CHartreeFockScfBatch(small, mode="grouped", stats=s1)
    scf.runX2CHartreeFockScfBatch(big, mode="grouped", stats=s3)
    assert s1["iterations"] == s3["iterations"]
    assert s3["launches_max_iteration"] == s1["launches_max_iteration"]
    assert s3["launches_total"] == s1["launches_total"]
    assert s3["autotune_seconds"] == 0.0
    _close(small)
    _close(big)


def test_non_projector_start_falls_back_to_the_recovery(ref_lib):
    systems = _systems([(24, 4), (30, 14)], seed0=360)
    # a start density with fractional occupations: not a projector, so the first iteration recovers
    # the occupied spinors instance by instance
    systems[1]["P0"] = 0.95 * systems[1]["P0"]
    probs = _problems(systems)
    st = {}
    batch = scf.runX2CHartreeFockScfBatch(probs, mode="grouped", stats=st)
    assert st["grouped_instances_first"] == 1
    for k, sy in enumerate(systems):
        rr = ref_lib.x2c_scf(sy)
        assert batch[k]["converged"] and abs(batch[k]["energy"] - rr["energy"]) <= 1e-8
    _close(probs)


def test_autotune_cache_round_trip(tmp_path):
    n = scf.autotune_cache()
    assert n > 0
    path = tmp_path / "tune.txt"
    scf.autotune_cache(save=path)
    lines = path.read_text().splitlines()
    assert len(lines) == n and all(len(line.split()) == 4 for line in lines)
    assert scf.autotune_cache(clear=True) == 0
    assert scf.autotune_cache(load=path) == n
