"""Building a Recipe from a TOML file or a plain table.

The steps and their order follow chadmv/plume src/plume/recipe/load.py:18-87: build the tables, check the
values the hot path depends on, apply --preview (coarser cells, preview frames, substeps raised so a step
keeps the full run's length), then fill the "empty means derived" defaults.
"""

import dataclasses
import difflib
import math
import re
import tomllib
import typing
from pathlib import Path

from plume_b200.recipe.errors import RecipeError
from plume_b200.recipe.schema import CHANNEL_LAYOUTS, FACE_KINDS, SEED_MAX, Recipe

# output names become file and folder names: one plain name, no path parts (recipe/rules.py:10-18)
PLAIN_NAME = re.compile(r"^[A-Za-z0-9_][A-Za-z0-9._-]*$")


def load_recipe(path: Path, preview: bool = False, sets=()) -> Recipe:
    """The recipe at `path`, merged over its `extends` parents, with `--set key=value` overrides applied
    (recipe/load.py:18-28, recipe/variation.py)."""
    from plume_b200.recipe.variation import apply_sets, read_toml, resolve_extends

    path = Path(path)
    table, _ = resolve_extends(read_toml(path), path)
    return resolve_table(apply_sets(table, sets), path.stem, preview)


def resolve_table(table: dict, recipe_stem: str, preview: bool = False) -> Recipe:
    recipe = parse_recipe(table)
    if preview:
        recipe = apply_preview(recipe)
    return fill_dependent_defaults(recipe, recipe_stem)


def parse_recipe(table: dict) -> Recipe:
    recipe = _build(Recipe, table, "")
    check_rules(recipe)
    return recipe


def apply_preview(recipe: Recipe) -> Recipe:
    preview = recipe.preview
    cell_m = max(recipe.domain.size_m) / preview.longest_axis_cells
    substeps = preview_substeps(recipe.time.frames, recipe.time.substeps, preview.frames)
    return dataclasses.replace(
        recipe,
        domain=dataclasses.replace(recipe.domain, cell_m=cell_m),
        time=dataclasses.replace(recipe.time, frames=preview.frames, substeps=substeps),
        output=dataclasses.replace(recipe.output, frame_px=preview.frame_px, columns=0))


def preview_substeps(frames: int, substeps: int, preview_frames: int) -> int:
    return max(1, math.ceil(frames * substeps / preview_frames))


def fill_dependent_defaults(recipe: Recipe, recipe_stem: str) -> Recipe:
    ambient = recipe.domain.ambient_k
    emitters = tuple(dataclasses.replace(e, temperature_k=ambient) if e.temperature_k == -1.0 else e
                     for e in recipe.emitter)
    output = recipe.output
    return dataclasses.replace(
        recipe, emitter=emitters,
        camera=dataclasses.replace(recipe.camera, seat=recipe.camera.seat or emitters[0].name),
        output=dataclasses.replace(output, name=output.name or recipe_stem,
                                   columns=output.columns or math.ceil(math.sqrt(recipe.time.frames))))


def check_rules(recipe: Recipe) -> None:
    """The value rules that protect the solver (a subset of chadmv/plume src/plume/recipe/rules.py:21-112)."""
    if not 0 <= recipe.seed <= SEED_MAX:
        raise RecipeError(f"seed must be between 0 and {SEED_MAX}, got {recipe.seed}")
    domain = recipe.domain
    if domain.cell_m <= 0 or any(size <= 0 for size in domain.size_m) or domain.ambient_k <= 0:
        raise RecipeError("domain.cell_m, domain.size_m and domain.ambient_k must be above 0")
    for name in ("bottom", "top", "left", "right", "back", "front"):
        if getattr(domain.faces, name) not in FACE_KINDS:
            raise RecipeError(f"domain.faces.{name} must be one of {', '.join(FACE_KINDS)}")
    time, solver = recipe.time, recipe.solver
    if time.duration_s <= 0 or time.frames < 1 or time.substeps < 1 or time.warmup_s < 0:
        raise RecipeError("time.duration_s must be above 0, frames and substeps at least 1, warmup_s at least 0")
    if not math.isfinite(time.frames * time.substeps / time.duration_s):
        raise RecipeError(f"time.duration_s is too small for {time.frames} frames, got {time.duration_s}")
    if solver.multigrid_cycles < 1 or solver.pressure_iterations < 1 or solver.max_substeps < 1:
        raise RecipeError("solver.multigrid_cycles, pressure_iterations and max_substeps must be at least 1")
    if solver.multigrid_sweeps < 2:
        raise RecipeError("solver.multigrid_sweeps must be at least 2 (one sweep a side diverges next to open "
                          "faces)")
    if solver.max_cells_per_step <= 0:
        raise RecipeError("solver.max_cells_per_step must be above 0")
    if not recipe.emitter:
        raise RecipeError("emitter needs at least one [[emitter]]")
    names = []
    for index, e in enumerate(recipe.emitter):
        if not e.name or any(mark in e.name for mark in ".[]"):  # key paths name emitters as emitter.<name>.<key>
            raise RecipeError(f"emitter[{index}].name must be a name without '.', '[' or ']'; got {e.name!r}")
        if e.name in names:
            raise RecipeError(f"emitter[{index}].name {e.name!r} is used twice")
        names.append(e.name)
        if e.shape == "sphere" and e.radius_m <= 0:
            raise RecipeError(f"emitter[{index}].radius_m must be above 0")
        if e.shape == "box" and any(size <= 0 for size in e.size_m):
            raise RecipeError(f"emitter[{index}].size_m must be above 0")
        if e.end_s <= e.start_s:
            raise RecipeError(f"emitter[{index}].end_s must be after start_s")
        if not 0.0 <= e.edge_softness <= 1.0:
            raise RecipeError(f"emitter[{index}].edge_softness must be between 0 and 1")
        if e.noise.scale_m <= 0 or e.noise.strength < 0 or e.smoke_per_s < 0:
            raise RecipeError(f"emitter[{index}] noise.scale_m must be above 0, noise.strength and "
                              f"smoke_per_s at least 0")
        _check_reaches_domain(domain.size_m, f"emitter[{index}]", e)
    if recipe.camera.seat and recipe.camera.seat not in names:
        raise RecipeError(f"camera.seat {recipe.camera.seat!r} is not an emitter; emitters are {', '.join(names)}")
    if recipe.output.name and (not PLAIN_NAME.match(recipe.output.name) or ".." in recipe.output.name):
        raise RecipeError(f"output.name must be a plain name of letters, digits, '.', '_' and '-'; got "
                          f"{recipe.output.name!r} (when output.name is empty the recipe's file name is used)")
    forces = recipe.forces
    if forces.drag_per_s < 0 or forces.vorticity_confinement < 0 or forces.turbulence.scale_m <= 0:
        raise RecipeError("forces.drag_per_s and vorticity_confinement must be at least 0, "
                          "turbulence.scale_m above 0")
    if any(forces.wind_mps) and forces.drag_per_s == 0.0:
        raise RecipeError("forces.wind_mps needs forces.drag_per_s above 0: drag is what pulls the gas toward "
                          "the wind")
    if recipe.output.channels not in CHANNEL_LAYOUTS:
        raise RecipeError(f"output.channels must be one of {', '.join(CHANNEL_LAYOUTS)}")


def _check_reaches_domain(size, where: str, emitter) -> None:
    """An emitter must reach into the domain (x and z span -size/2..size/2, y 0..size); its centre may lie
    outside, as a source half sunk below the floor does (recipe/rules.py:86-99)."""
    ranges = ((-size[0] / 2, size[0] / 2), (0.0, size[1]), (-size[2] / 2, size[2] / 2))
    reaches = (emitter.radius_m,) * 3 if emitter.shape == "sphere" else tuple(s / 2 for s in emitter.size_m)
    for axis, centre, reach, (low, high) in zip("xyz", emitter.center_m, reaches, ranges):
        if centre - reach > high or centre + reach < low:
            raise RecipeError(f"{where} lies outside the domain on {axis}: its center {centre:g} m reaches "
                              f"{reach:g} m, and the domain spans {low:g} to {high:g} m")


def _build(cls: type, table: dict, where: str):
    if not isinstance(table, dict):
        raise RecipeError(f"{where or 'recipe'} must be a table")
    hints = typing.get_type_hints(cls)
    fields = {f.name: f for f in dataclasses.fields(cls)}
    for key in table:
        if key not in fields and not (where == "" and key == "resolved") and not (where == "look" and
                                                                                key == "backgrounds"):
            close = difflib.get_close_matches(key, list(fields), n=1)
            hint = f"; did you mean {close[0]}?" if close else ""
            raise RecipeError(f"unknown key {where + '.' if where else ''}{key}{hint}")
    values = {}
    for name, f in fields.items():
        path = f"{where}.{name}" if where else name
        if name not in table:
            if f.default is dataclasses.MISSING and f.default_factory is dataclasses.MISSING:
                raise RecipeError(f"{path} is required")
            continue
        values[name] = _convert(table[name], hints[name], path)
    return cls(**values)


def _convert(value, annotation, path: str):
    if dataclasses.is_dataclass(annotation):
        return _build(annotation, value, path)
    if annotation is float:
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise RecipeError(f"{path} must be a number, got {value!r}")
        try:
            number = float(value)
        except OverflowError:  # a whole number beyond the float range
            number = math.inf
        if not math.isfinite(number):  # nan and inf would pass every range rule and fail deep in a run
            raise RecipeError(f"{path} must be a finite number, got {number}")
        return number
    if annotation is int:
        if isinstance(value, bool) or not isinstance(value, int):
            raise RecipeError(f"{path} must be a whole number, got {value!r}")
        return value
    if annotation is str:
        if not isinstance(value, str):
            raise RecipeError(f"{path} must be text, got {value!r}")
        return value
    args = typing.get_args(annotation)
    if not isinstance(value, list):
        hint = f" (write [[{path}]] for each one)" if isinstance(value, dict) else ""
        raise RecipeError(f"{path} must be a list, got {value!r}{hint}")
    if len(args) == 2 and args[1] is Ellipsis:
        return tuple(_convert(item, args[0], f"{path}[{i}]") for i, item in enumerate(value))
    if len(value) != len(args):
        raise RecipeError(f"{path} must have {len(args)} values, got {len(value)}")
    return tuple(_convert(item, kind, f"{path}[{i}]") for i, (item, kind) in enumerate(zip(value, args)))
