"""Values computed from a resolved recipe: cell counts, the rounded domain, and the step timing.

Same formulas as chadmv/plume src/plume/recipe/derived.py:23-38 (cells round size/cell, the domain's origin is
the centre of its floor, dt = 1 / (fps * substeps)).
"""

from dataclasses import dataclass

from plume_b200.recipe.schema import Recipe


@dataclass(frozen=True)
class Derived:
    cells: tuple[int, int, int]
    size_m: tuple[float, float, float]
    domain_min_m: tuple[float, float, float]
    fps: float
    dt_s: float
    warmup_steps: int
    steps_per_frame: int

    def frame_time_s(self, frame: int) -> float:
        return (frame + 1) / self.fps


def derive(recipe: Recipe) -> Derived:
    cell = recipe.domain.cell_m
    cells = tuple(max(1, round(extent / cell)) for extent in recipe.domain.size_m)
    size = tuple(n * cell for n in cells)
    fps = recipe.time.frames / recipe.time.duration_s
    dt = 1.0 / (fps * recipe.time.substeps)
    return Derived(cells=cells, size_m=size, domain_min_m=(-size[0] / 2, 0.0, -size[2] / 2), fps=fps, dt_s=dt,
                   warmup_steps=round(recipe.time.warmup_s / dt), steps_per_frame=recipe.time.substeps)
