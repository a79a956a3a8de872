"""Recipe variations (mirrors chadmv/plume src/plume/recipe/variation.py): `extends` (a recipe built on a
parent recipe file) and `--set key=value` overrides, both applied to the parsed TOML table before the schema
builds it, so every key they bring in meets the same strict checks as a key written in the file.

A sweep of variations of one recipe (preview variants, parameter sweeps) is the batched runner's input:
`sweep` resolves one recipe per list of overrides.
"""

import copy
import re
import tomllib
from pathlib import Path, PurePosixPath, PureWindowsPath

from plume_b200.recipe.errors import RecipeError

MAX_EXTENDS_DEPTH = 8
_INDEXED_EMITTER = re.compile(r"^emitter\[(\d+)\]$")


def read_toml(path: Path) -> dict:
    try:
        with Path(path).open("rb") as handle:
            return tomllib.load(handle)
    except FileNotFoundError:
        raise RecipeError(f"recipe not found: {path}") from None
    except (tomllib.TOMLDecodeError, UnicodeDecodeError) as error:
        raise RecipeError(f"{path} is not valid TOML: {error}") from None


def deep_merge(parent: dict, child: dict) -> dict:
    """The child's values over the parent's: tables merge key by key, anything else (lists included) is
    replaced whole, so a child's [[emitter]] list replaces the parent's."""
    merged = dict(parent)
    for key, value in child.items():
        merged[key] = deep_merge(merged[key], value) if isinstance(value, dict) and isinstance(merged.get(key), dict) \
            else value
    return merged


def _check_parent_path(text: str) -> None:
    if PurePosixPath(text).is_absolute() or PureWindowsPath(text).is_absolute() or PureWindowsPath(text).drive:
        raise RecipeError(f"extends must be a path relative to the recipe, got {text!r}")
    if not text.endswith(".toml"):
        raise RecipeError(f"extends must name a .toml recipe, got {text!r}")


def resolve_extends(table: dict, path: Path) -> tuple[dict, tuple[str, ...]]:
    """The table merged over its parents (each named relative to its child), and the parents as written."""
    path = Path(path)
    chain, seen, merged, child = [], {path.resolve()}, dict(table), path
    while True:
        parent_text = merged.pop("extends", "")
        if not isinstance(parent_text, str):
            raise RecipeError(f"extends in {child} must be text")
        if not parent_text:
            return merged, tuple(chain)
        _check_parent_path(parent_text)
        if len(chain) == MAX_EXTENDS_DEPTH:
            raise RecipeError(f"extends goes deeper than {MAX_EXTENDS_DEPTH} parents, starting at {path}")
        parent_path = child.parent / parent_text
        if parent_path.resolve() in seen:
            raise RecipeError(f"extends forms a loop: {child} extends {parent_text}, already in the chain")
        seen.add(parent_path.resolve())
        chain.append(parent_text)
        merged = deep_merge(read_toml(parent_path), merged)
        child = parent_path


def _parse_value(text: str):
    try:
        return tomllib.loads(f"value = {text}")["value"]
    except tomllib.TOMLDecodeError:
        return text  # plain text, so domain.faces.top=closed works


def set_item(item: str):
    key, sep, value = item.partition("=")
    key = key.strip()
    if not sep or not key:
        raise RecipeError(f"--set needs key=value, got {item!r}")
    if key == "extends":
        raise RecipeError("--set cannot change extends; parents are merged before --set applies")
    return key, _parse_value(value.strip())


def _emitter(table: dict, parts: list, index: int, label: str):
    emitters = table.get("emitter")
    if not isinstance(emitters, list) or not emitters:
        raise RecipeError(f"{label}: the recipe has no [[emitter]]")
    match = _INDEXED_EMITTER.match(parts[index])
    if match:
        position = int(match.group(1))
        if position >= len(emitters):
            raise RecipeError(f"{label}: emitter[{position}] does not exist; the recipe has {len(emitters)}")
        return emitters[position], index + 1
    if len(parts) < index + 3:
        raise RecipeError(f"{label}: name the emitter, as emitter.<name>.<key> or emitter[0].<key>")
    names = [e.get("name") if isinstance(e, dict) else None for e in emitters]
    if parts[index + 1] not in names:
        raise RecipeError(f"{label}: no emitter is named {parts[index + 1]!r}; emitters are "
                          f"{', '.join(str(n) for n in names)}")
    return emitters[names.index(parts[index + 1])], index + 2


def _set_value(table: dict, key: str, value, label: str) -> None:
    parts = key.split(".")
    target, index = table, 0
    while index < len(parts) - 1:
        part = parts[index]
        if part == "emitter" or _INDEXED_EMITTER.match(part):
            target, index = _emitter(table, parts, index, label)
            continue
        child = target.setdefault(part, {})
        if not isinstance(child, dict):
            raise RecipeError(f"{label}: {'.'.join(parts[:index + 1])} is a value, not a table")
        target, index = child, index + 1
    target[parts[-1]] = value


def apply_sets(table: dict, sets) -> dict:
    """A copy of the table with each `key=value` override applied in order (dotted keys; an emitter by name,
    emitter.<name>.<key>, or index, emitter[0].<key>; values read as TOML, else as plain text)."""
    result = copy.deepcopy(table)
    for item in sets:
        key, value = set_item(item)
        _set_value(result, key, value, f"--set {item!r}")
    return result


def sweep(path: Path, variations, preview: bool = False) -> list:
    """One resolved recipe per list of `key=value` overrides of the recipe at `path` (the batched runner's
    instances)."""
    from plume_b200.recipe.load import load_recipe

    return [load_recipe(path, preview=preview, sets=tuple(sets)) for sets in variations]


def sweep_table(table: dict, variations, stem: str = "sweep", preview: bool = False) -> list:
    """`sweep` of a recipe already parsed from TOML (extends resolved): instance n is the table with the n-th
    list of overrides applied, named `<stem>_<n>`."""
    from plume_b200.recipe.load import resolve_table

    return [resolve_table(apply_sets(table, tuple(sets)), f"{stem}_{n}", preview) for n, sets in enumerate(variations)]
