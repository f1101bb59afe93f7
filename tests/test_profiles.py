"""The committed ncu summaries that bench.py reads for its roofline fields
(profiles/instruction_mix.json for the step's issue and FP64 floors,
profiles/ncu_traffic.json for the dominant kernel's DRAM traffic) parse, and
cover every kernel class of the C2 step that the bench can name as dominant."""
import json
import pathlib

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
STEP_CLASSES = ["advect_x", "advect_y", "advect_z", "cn_solve_x", "cn_solve_y", "cn_solve_z", "totals"]
CELL_GRAINS_C2 = 720 * 360 * 60 * 10


def _load(name):
    return json.loads((ROOT / "profiles" / name).read_text())


def test_instruction_mix_covers_the_step():
    mix = _load("instruction_mix.json")["C2"]
    assert set(STEP_CLASSES) <= set(mix)
    for k in STEP_CLASSES:
        inst, fp64 = mix[k]["thread_inst_per_cg"], mix[k]["fp64_inst_per_cg"]
        assert 0 < fp64 < inst < 1000, (k, inst, fp64)


def test_traffic_covers_the_step():
    traffic = _load("ncu_traffic.json")["C2"]
    assert set(STEP_CLASSES) <= set(traffic)
    level = 8.0 * CELL_GRAINS_C2  # one concentration level of C2, bytes
    for k in STEP_CLASSES:
        # every one of these kernels reads a level at least once and moves at
        # most a few levels
        assert 0.9 * level <= traffic[k] <= 4.0 * level, (k, traffic[k] / level)


def test_bench_floors_from_the_summaries():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    fl = bench.compute_floors("C2", CELL_GRAINS_C2)
    assert fl is not None
    # the FP64-pipe floor lies below the issue floor, and both below any
    # measured C2 step (several ms)
    assert 0 < fl["fp64_floor_ms"] < fl["issue_floor_ms"] < 6.0
    assert bench.ncu_traffic("C2", "advect_x") == pytest.approx(_load("ncu_traffic.json")["C2"]["advect_x"])
