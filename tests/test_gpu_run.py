"""The smoke-puff preview run end to end on the device (simulate, render, sheet, numbers), against the
reference's approved numbers file with the reference's golden tolerances (tests/cli/test_golden_numbers.py in
chadmv/plume): amounts within 2% (floor 1e-3), box edges and heat within 0.02, peak and fade frames within
one frame; and a second run gives identical bytes (tests/cli/test_gpu_same_bytes.py)."""

import importlib.util
from pathlib import Path

import pytest

from support import host

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_tools():
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def preview_run():
    from plume_b200.recipe.load import load_recipe
    from plume_b200.run import run_recipe

    return run_recipe(load_recipe(GOLDEN / "smoke_puff.toml", preview=True), "recipes/smoke_puff.toml")


def test_the_preview_run_matches_the_golden_numbers(cuda_device):
    tools = golden_tools()
    run = preview_run()
    golden = (GOLDEN / "smoke_puff_preview.numbers.txt").read_text()
    assert run.steps.total_steps == 192
    assert tools.numbers_close(run.numbers, golden) == []
    actual, _ = tools.read_numbers(run.numbers)
    expected, _ = tools.read_numbers(golden)
    assert actual["recipe"] == expected["recipe"] and actual["channels"] == expected["channels"]
    for key in ("fps", "frame_m"):
        assert float(actual[key]) == pytest.approx(float(expected[key]), rel=1e-6), key


def test_two_preview_runs_give_identical_bytes(cuda_device):
    first, second = preview_run(), preview_run()
    assert first.numbers == second.numbers
    assert host(first.sheet).tobytes() == host(second.sheet).tobytes()
    assert host(first.raw).tobytes() == host(second.raw).tobytes()
