"""The oracle is pinned to the reference: its FP32 raw frames reproduce the reference's own SHA-256 digests
(Warp 1.19 CPU, Linux) byte for byte, and its smoke puff preview reproduces the reference's golden numbers file
through the reference's own sheet and report code (when the reference is mounted)."""

import copy
import hashlib
import json
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.recipe.derived import derive
from plume_b200.recipe.load import resolve_table
from plume_b200.render.camera import make_camera, make_domain_view

GOLDEN = Path(__file__).resolve().parent / "golden"
REFERENCE = Path(os.environ.get("PLUME_REFERENCE", "/root/reference"))
DIGESTS = json.loads((GOLDEN / "raw_frame_digests.json").read_text())


@pytest.mark.parametrize("channels", sorted(DIGESTS["digests"]))
def test_oracle_reproduces_the_reference_raw_frame_digest(channels):
    table = copy.deepcopy(DIGESTS["recipe"])
    table["output"] = {"channels": channels}
    recipe = resolve_table(table, "tiny")
    derived = derive(recipe)
    view = make_domain_view(make_camera(20.0, 30.0), derived.domain_min_m, derived.size_m, recipe.domain.cell_m,
                            recipe.render.px_per_cell)
    renderer = O.FrameRenderer(view, recipe.render, derived.cells, channels)
    frames = []
    O.simulate(recipe, derived, lambda frame, grid: frames.append(renderer.render(grid)))
    frame = frames[-1].astype(np.float32)
    assert list(frame.shape) == DIGESTS["shape"]
    assert hashlib.sha256(frame.tobytes()).hexdigest() == DIGESTS["digests"][channels]


@pytest.mark.skipif(not (REFERENCE / "src" / "plume").exists(), reason="the reference is not mounted")
def test_oracle_preview_matches_the_reference_golden_numbers():
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    make_golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(make_golden)
    _, _, frames, log = make_golden.oracle_preview_frames()
    assert log.total_steps == 192
    text = make_golden.reference_numbers(frames)
    assert make_golden.numbers_close(text, (GOLDEN / "smoke_puff_preview.numbers.txt").read_text()) == []
    stats = json.loads((GOLDEN / "preview_raw_stats.json").read_text())
    assert make_golden.raw_stats(frames)["sum"] == stats["sum"]
