"""The sheet oracle is pinned to the reference: its bicubic resampling is Pillow's, bit for bit, and its
assembly of the smoke puff preview's raw frames reproduces the reference's own sheet digests
(tests/golden/preview_sheet.json, written by make_golden.py with the reference's sheet code) in both layouts.
The product's tap tables equal the oracle's."""

import importlib.util
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import sheet as S

GOLDEN = Path(__file__).resolve().parent / "golden"


def make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def test_resampling_is_pillows_bicubic_bit_for_bit():
    from PIL import Image

    rng = np.random.default_rng(7)
    for _ in range(25):
        h, w = (int(x) for x in rng.integers(10, 200, 2))
        plane = (rng.standard_normal((h, w)) * rng.choice([1.0, 500.0])).astype(np.float32)
        out = int(rng.integers(4, 180))
        x0, y0 = float(rng.uniform(0, w / 2)), float(rng.uniform(0, h / 2))
        side = float(rng.uniform(1, min(w - x0, h - y0)))
        box = (x0, y0, x0 + side, y0 + side)
        expected = np.asarray(Image.fromarray(plane).resize((out, out), Image.Resampling.BICUBIC, box=box))
        assert np.array_equal(S.resample_plane(plane, box, out), expected), (h, w, out, box)


def test_product_tap_tables_equal_the_oracle():
    from plume_b200.sheet.resample import taps

    rng = np.random.default_rng(3)
    for _ in range(100):
        n, out = int(rng.integers(5, 400)), int(rng.integers(2, 300))
        a = float(rng.uniform(0, n / 2))
        b = float(rng.uniform(a + 0.5, n))
        first, count, weights = S.coefficients(n, a, b, out)
        t = taps(n, a, b, out)
        assert np.array_equal(first, t.first) and np.array_equal(count, t.count) and np.array_equal(weights, t.weights)


@pytest.fixture(scope="module")
def preview():
    recipe, derived, frames, _ = make_golden().oracle_preview_frames()
    return recipe, derived, frames


def test_oracle_sheet_reproduces_the_reference_sheet(preview):
    recipe, _, frames = preview
    golden = json.loads((GOLDEN / "preview_sheet.json").read_text())["layouts"]
    digest = make_golden().frames_digest
    for layout, want in golden.items():
        quantized, crop, margin, heat_divisor, shade_divisor = S.assemble(frames, recipe.output.frame_px,
                                                                          recipe.render, layout)
        assert list(crop) == want["crop"] and margin == want["margin"]
        assert heat_divisor == want["heat_divisor"] and shade_divisor == want["shade_divisor"]
        assert digest(quantized) == want["frames_sha256"], layout


def test_numbers_text_of_the_oracle_sheet_is_the_reference_numbers_file(preview):
    from plume_b200.sheet.numbers import FrameNumbers, RunFacts, numbers_text

    recipe, derived, frames = preview
    quantized, crop, _, heat_divisor, shade_divisor = S.assemble(frames, recipe.output.frame_px, recipe.render,
                                                                 recipe.output.channels)
    rows = []
    for index, frame in enumerate(quantized):
        coverage, box, mean_heat, mean_thick, total_thick, peak_heat = S.measure_frame(frame)
        rows.append(FrameNumbers(index, (index + 1) / derived.fps, coverage, box, mean_heat, mean_thick, total_thick,
                                 peak_heat))
    from plume_b200.render.camera import sheet_domain_view

    view = sheet_domain_view(recipe, derived)
    nx, ny, nz = derived.cells
    facts = RunFacts(recipe="recipes/smoke_puff.toml", backend="cpu",
                     grid=f"{nx} x {ny} x {nz} cells of {recipe.domain.cell_m:.6f} m", fps=derived.fps,
                     frame_m=crop[2] * view.pixel_m, heat_divisor=heat_divisor, channels=recipe.output.channels,
                     shade_divisor=shade_divisor)
    assert numbers_text(rows, facts) == (GOLDEN / "oracle_preview.numbers.txt").read_text()
