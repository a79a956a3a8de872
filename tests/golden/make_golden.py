"""Regenerates the oracle's golden fixtures and pins the oracle against the reference.

Run from the repository root, in a container where chadmv/plume is mounted at /root/reference (or at $PLUME_REFERENCE):

    python tests/golden/make_golden.py

It runs the smoke puff preview (38 x 48 x 38 cells, 16 frames, 192 substeps) through the FP32 oracle, turns
the raw frames into the sheet and numbers file with the reference's own host code (`plume.sheet.assemble`,
`plume.report.numbers`, importable without Warp), checks the numbers against the reference's golden file
(`tests/golden/smoke_puff_preview.numbers.txt`, copied here) with the reference's tolerances
(tests/cli/test_golden_numbers.py:148-188), and writes:

    preview_raw_stats.json          per-frame sums and maxima of the oracle's raw frames
    oracle_preview.numbers.txt      the numbers file the reference's sheet code makes of those frames

The GPU tests compare the CUDA path's raw frames with the oracle run on the same host and with these
statistics; they never read the reference.
"""

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REFERENCE_SRC = Path(os.environ.get("PLUME_REFERENCE", "/root/reference")) / "src"
sys.path.insert(0, str(REPO))

from oracle import oracle as O  # noqa: E402
from plume_b200.recipe.derived import derive  # noqa: E402
from plume_b200.recipe.load import load_recipe  # noqa: E402
from plume_b200.render.camera import sheet_domain_view  # noqa: E402


def oracle_preview_frames():
    recipe = load_recipe(HERE / "smoke_puff.toml", preview=True)
    derived = derive(recipe)
    view = sheet_domain_view(recipe, derived)
    renderer = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels)
    frames = []
    log = O.simulate(recipe, derived, lambda frame, grid: frames.append(renderer.render(grid)))
    return recipe, derived, frames, log


def raw_stats(frames) -> dict:
    return {"sum": [[float(x) for x in f.astype(np.float64).sum(axis=(0, 1))] for f in frames],
            "max": [[float(x) for x in f.max(axis=(0, 1))] for f in frames],
            "shape": list(frames[0].shape)}


def reference_numbers(frames) -> str:
    sys.path.insert(0, str(REFERENCE_SRC))
    from plume.recipe.derived import derive as ref_derive
    from plume.recipe.load import load_recipe as ref_load
    from plume.render.camera import sheet_domain_view as ref_view
    from plume.report.numbers import RunFacts, measure, numbers_text
    from plume.sheet.assemble import assemble, seat_point

    recipe = ref_load(HERE / "smoke_puff.toml", preview=True)
    derived = ref_derive(recipe)
    view = ref_view(recipe, derived)
    assembled = assemble(list(frames), view, seat_point(recipe), recipe.output.frame_px, recipe.render,
                         recipe.output.channels)
    nx, ny, nz = derived.cells
    facts = RunFacts(recipe="recipes/smoke_puff.toml", backend="cpu",
                     grid=f"{nx} x {ny} x {nz} cells of {recipe.domain.cell_m:.6f} m", fps=derived.fps,
                     frame_m=assembled.frame_m, heat_divisor=assembled.heat_divisor, channels=recipe.output.channels,
                     shade_divisor=assembled.shade_divisor)
    return numbers_text(measure(assembled.frames, derived.fps), facts)


LAYOUTS = ("heat,thickness,shade,unused", "heat,thickness,normal_x,normal_y")


def frames_digest(frames) -> str:
    digest = hashlib.sha256()
    for frame in frames:
        digest.update(np.ascontiguousarray(frame, dtype=np.uint8).tobytes())
    return digest.hexdigest()


def reference_sheets(frames) -> dict:
    """The reference's own sheet assembly (plume.sheet.assemble) of the oracle's preview frames, in both
    channel layouts: the crop, margin, divisors and a SHA-256 of the quantised frames."""
    sys.path.insert(0, str(REFERENCE_SRC))
    from plume.recipe.derived import derive as ref_derive
    from plume.recipe.load import load_recipe as ref_load
    from plume.render.camera import sheet_domain_view as ref_view
    from plume.sheet.assemble import assemble, seat_point

    recipe = ref_load(HERE / "smoke_puff.toml", preview=True)
    view = ref_view(recipe, ref_derive(recipe))
    sheets = {}
    for layout in LAYOUTS:
        a = assemble(list(frames), view, seat_point(recipe), recipe.output.frame_px, recipe.render, layout)
        sheets[layout] = {"crop": [a.crop.left, a.crop.top, a.crop.side], "margin": a.margin,
                          "heat_divisor": a.heat_divisor, "shade_divisor": a.shade_divisor,
                          "frames_sha256": frames_digest(a.frames)}
    return sheets


def read_numbers(text: str):
    head, _, table = text.partition("\n\n")
    summary = {}
    for line in head.splitlines():
        key, _, value = line.partition(" ")
        summary[key] = value.strip()
    lines = table.strip().splitlines()
    names = lines[0].split()
    return summary, [dict(zip(names, line.split())) for line in lines[1:]]


def numbers_close(actual: str, golden: str) -> list[str]:
    """Differences beyond the reference's golden tolerances (empty when the numbers agree)."""
    problems = []
    a_summary, a_rows = read_numbers(actual)
    g_summary, g_rows = read_numbers(golden)
    for key in ("grid", "frames"):
        if a_summary[key] != g_summary[key]:
            problems.append(f"summary {key}: {a_summary[key]} != {g_summary[key]}")
    for key in ("peak_frame", "fade_frame"):
        if (a_summary[key] == "never") != (g_summary[key] == "never") or (
                g_summary[key] != "never" and abs(int(a_summary[key]) - int(g_summary[key])) > 1):
            problems.append(f"summary {key}: {a_summary[key]} != {g_summary[key]}")
    if len(a_rows) != len(g_rows):
        return problems + [f"{len(a_rows)} rows != {len(g_rows)}"]
    for a, g in zip(a_rows, g_rows):
        for key in ("left", "top", "right", "bottom"):
            if (a[key] == "-") != (g[key] == "-") or (g[key] != "-" and abs(float(a[key]) - float(g[key])) > 0.02):
                problems.append(f"frame {g['frame']} {key}: {a[key]} != {g[key]}")
        for key in ("coverage", "mean_thick", "total_thick"):
            x, y = float(a[key]), float(g[key])
            if abs(x - y) > max(0.02 * abs(y), 1e-3):
                problems.append(f"frame {g['frame']} {key}: {a[key]} != {g[key]}")
        for key in ("mean_heat", "peak_heat"):
            if abs(float(a[key]) - float(g[key])) > 0.02:
                problems.append(f"frame {g['frame']} {key}: {a[key]} != {g[key]}")
    return problems


def main() -> None:
    recipe, derived, frames, log = oracle_preview_frames()
    stats = raw_stats(frames)
    stats["steps_per_frame"] = list(log.steps_per_frame)
    (HERE / "preview_raw_stats.json").write_text(json.dumps(stats, indent=1) + "\n")
    if not REFERENCE_SRC.exists():
        print("reference not mounted: wrote raw statistics only")
        return
    text = reference_numbers(frames)
    (HERE / "oracle_preview.numbers.txt").write_text(text)
    sheets = {"source": "chadmv/plume src/plume/sheet/assemble.py:39-60 (reference code, run on the oracle's "
                        "smoke puff preview raw frames)", "layouts": reference_sheets(frames)}
    (HERE / "preview_sheet.json").write_text(json.dumps(sheets, indent=1) + "\n")
    problems = numbers_close(text, (HERE / "smoke_puff_preview.numbers.txt").read_text())
    print("golden numbers:", "match within the reference's tolerances" if not problems else problems)
    if problems:
        raise SystemExit(1)


if __name__ == "__main__":
    main()
