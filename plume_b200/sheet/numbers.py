"""Per-frame measurements of the quantised sheet frames on the device (mirrors chadmv/plume
src/plume/report/numbers.py:42-100). The device tallies integers per frame (covered count and box, byte sums,
largest heat byte); the host turns them into the reference's FrameNumbers and text."""

from dataclasses import dataclass

import numpy as np
import torch

from plume_b200 import _native as N

COVERED_LEVEL = 8  # numbers.py:10
FADE_FRACTION = 0.1
KEY_WIDTH = 18
COLUMNS = ("frame", "time_s", "coverage", "left", "top", "right", "bottom", "mean_heat", "mean_thick",
           "total_thick", "peak_heat")
WIDTHS = (5, 8, 9, 7, 7, 7, 7, 10, 11, 12, 10)
MEASURE_FIELDS = 9


@dataclass(frozen=True)
class FrameNumbers:
    frame: int
    time_s: float
    coverage: float
    box: tuple | None
    mean_heat: float
    mean_thick: float
    total_thick: float
    peak_heat: float


@dataclass(frozen=True)
class RunFacts:
    recipe: str
    backend: str
    grid: str
    fps: float
    frame_m: float
    heat_divisor: float
    channels: str
    shade_divisor: float | None


def measure(frames: torch.Tensor, fps: float) -> list[FrameNumbers]:
    """Per-frame measurements of (frames, size, size, 4) uint8 frames on the device."""
    count, size = frames.shape[0], frames.shape[1]
    stats = torch.empty((count, MEASURE_FIELDS), dtype=torch.int64, device=frames.device)
    N.call("plume_sheet_measure", N.ptr(frames.contiguous(), torch.uint8), count, size, COVERED_LEVEL,
           N.ptr(stats, torch.int64), N.stream())
    rows = []
    for index, s in enumerate(stats.cpu().numpy().tolist()):
        covered, left, top, right, bottom, heat_sum, thick_sum, thick_total, heat_peak = s
        box = (left / size, top / size, right / size, bottom / size) if covered else None
        rows.append(FrameNumbers(
            frame=index, time_s=(index + 1) / fps, coverage=covered / (size * size), box=box,
            mean_heat=heat_sum / 255.0 / covered if covered else 0.0,
            mean_thick=thick_sum / 255.0 / covered if covered else 0.0,
            total_thick=thick_total / 255.0, peak_heat=heat_peak / 255.0))
    return rows


def peak_and_fade(rows):
    totals = [row.total_thick for row in rows]
    peak = int(np.argmax(totals))
    for row in rows[peak + 1:]:
        if row.total_thick < FADE_FRACTION * totals[peak]:
            return peak, row.frame
    return peak, None


def numbers_text(rows, facts: RunFacts) -> str:
    """The numbers file's text (numbers.py:57-77)."""
    peak, fade = peak_and_fade(rows)
    summary = [
        ("recipe", facts.recipe), ("backend", facts.backend), ("grid", facts.grid), ("frames", str(len(rows))),
        ("fps", f"{facts.fps:.6f}"), ("frame_m", f"{facts.frame_m:.6f}"),
        ("heat_divisor", f"{facts.heat_divisor:.6f} K m"), ("channels", facts.channels),
        *([("shade_divisor", f"{facts.shade_divisor:.6f}")] if facts.shade_divisor is not None else []),
        ("peak_frame", str(peak)), ("fade_frame", "never" if fade is None else str(fade)),
    ]
    lines = [f"{key:<{KEY_WIDTH}}{value}" for key, value in summary]
    lines.append("")
    lines.append(_row_text(COLUMNS))
    for row in rows:
        box = [f"{value:.4f}" for value in row.box] if row.box else ["-"] * 4
        lines.append(_row_text([str(row.frame), f"{row.time_s:.4f}", f"{row.coverage:.4f}", *box,
                                f"{row.mean_heat:.4f}", f"{row.mean_thick:.4f}", f"{row.total_thick:.4f}",
                                f"{row.peak_heat:.4f}"]))
    return "\n".join(lines) + "\n"


def _row_text(values) -> str:
    return " ".join(f"{value:>{width}}" for value, width in zip(values, WIDTHS)).rstrip()
