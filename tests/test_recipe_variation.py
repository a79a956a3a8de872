"""Recipe variations as the reference defines them (its tests/recipe/test_variation.py:42-157): `extends`
chains merged table by table, `--set` overrides of numbers, vectors, text and emitters, and the errors for
malformed ones; and a sweep of variations resolves one recipe per override list (the batched runner's input)."""

import tomllib

import pytest

from plume_b200.recipe.errors import RecipeError
from plume_b200.recipe.load import load_recipe
from plume_b200.recipe.variation import apply_sets, sweep

PARENT = """
seed = 4

[domain]
size_m = [2.0, 3.0, 2.0]
cell_m = 0.1
faces = { top = "open", left = "closed" }

[time]
duration_s = 2.0

[[emitter]]
name = "puff"
center_m = [0.0, 0.3, 0.0]
radius_m = 0.25
end_s = 0.25
smoke_per_s = 4.0
noise = { scale_m = 0.2, strength = 0.5 }

[dissipation]
smoke_per_s = 1.0
"""


def write(folder, name, text):
    folder.mkdir(parents=True, exist_ok=True)
    path = folder / name
    path.write_text(text)
    return path


def test_child_overrides_one_key_and_inherits_the_rest(tmp_path):
    write(tmp_path, "base.toml", PARENT)
    child = write(tmp_path, "child.toml", 'extends = "base.toml"\n[dissipation]\nsmoke_per_s = 2.5\n')
    recipe = load_recipe(child)
    assert (recipe.dissipation.smoke_per_s, recipe.seed, recipe.emitter[0].smoke_per_s) == (2.5, 4, 4.0)
    assert recipe.extends == "" and recipe.output.name == "child"


def test_nested_tables_merge_and_emitter_lists_replace(tmp_path):
    write(tmp_path, "base.toml", PARENT)
    child = write(tmp_path, "child.toml", 'extends = "base.toml"\n[domain.faces]\nright = "closed"\n')
    faces = load_recipe(child).domain.faces
    assert (faces.left, faces.right, faces.top) == ("closed", "closed", "open")
    other = write(tmp_path, "other.toml", 'extends = "base.toml"\n[[emitter]]\nname = "other"\n'
                                          'center_m = [0.0, 0.5, 0.0]\nradius_m = 0.1\nend_s = 0.5\n')
    assert [e.name for e in load_recipe(other).emitter] == ["other"]


def test_grandparent_chain_resolves_relative_to_each_file(tmp_path):
    write(tmp_path / "shared", "base.toml", PARENT)
    write(tmp_path / "shared", "middle.toml", 'extends = "base.toml"\nseed = 9\n')
    child = write(tmp_path / "effects", "child.toml", 'extends = "../shared/middle.toml"\n[time]\nframes = 32\n')
    recipe = load_recipe(child)
    assert (recipe.seed, recipe.time.frames, recipe.time.duration_s) == (9, 32, 2.0)


@pytest.mark.parametrize("text, message", [
    ('extends = "b.toml"\n', "loop"), ("extends = '/etc/base.toml'\n", "relative"),
    ("extends = 'C:base.toml'\n", "relative"), ('extends = "base.txt"\n', ".toml"),
    ('extends = "missing.toml"\n', "missing.toml")])
def test_bad_parents_fail(tmp_path, text, message):
    write(tmp_path, "b.toml", 'extends = "a.toml"\n')
    path = write(tmp_path, "a.toml", text)
    with pytest.raises(RecipeError, match=message):
        load_recipe(path)


def test_set_overrides_numbers_vectors_text_and_emitters(tmp_path):
    path = write(tmp_path, "base.toml", PARENT)
    recipe = load_recipe(path, sets=("dissipation.cooling_per_s=0.5", "emitter.puff.velocity_mps=[0, 1.5, 0]",
                                     "emitter[0].radius_m = 0.4", "emitter.puff.noise.strength=0.9",
                                     "domain.faces.top=closed", "output.name=variant"))
    assert recipe.dissipation.cooling_per_s == 0.5
    assert recipe.emitter[0].velocity_mps == (0.0, 1.5, 0.0)
    assert recipe.emitter[0].radius_m == 0.4 and recipe.emitter[0].noise.strength == 0.9
    assert recipe.domain.faces.top == "closed" and recipe.output.name == "variant"


def test_set_applies_after_extends_and_names_the_closest_key(tmp_path):
    write(tmp_path, "base.toml", PARENT)
    child = write(tmp_path, "child.toml", 'extends = "base.toml"\nseed = 5\n')
    assert load_recipe(child, sets=("seed=6",)).seed == 6
    with pytest.raises(RecipeError, match="did you mean cooling_per_s"):
        load_recipe(child, sets=("dissipation.cooling_per=0.5",))


@pytest.mark.parametrize("item, message", [
    ("seed", "key=value"), ("emitter.nobody.radius_m=1", "no emitter is named 'nobody'"),
    ("emitter[3].radius_m=1", r"emitter\[3\] does not exist"), ("emitter.puff=1", "name the emitter"),
    ("seed.x=1", "is a value, not a table"), ("extends=other.toml", "cannot change extends")])
def test_malformed_sets_fail(tmp_path, item, message):
    path = write(tmp_path, "base.toml", PARENT)
    with pytest.raises(RecipeError, match=message):
        load_recipe(path, sets=(item,))


def test_set_leaves_the_parsed_table_unchanged():
    table = tomllib.loads(PARENT)
    apply_sets(table, ("emitter.puff.noise.strength=0.1", "domain.faces.top=closed"))
    assert table["emitter"][0]["noise"]["strength"] == 0.5 and table["domain"]["faces"]["top"] == "open"


def test_a_sweep_resolves_one_recipe_per_variation(tmp_path):
    path = write(tmp_path, "base.toml", PARENT)
    recipes = sweep(path, [(), ("forces.drag_per_s=0.3",), ("emitter.puff.radius_m=0.4", "seed=11")], preview=True)
    assert [r.forces.drag_per_s for r in recipes] == [0.0, 0.3, 0.0]
    assert [r.emitter[0].radius_m for r in recipes] == [0.25, 0.25, 0.4] and recipes[2].seed == 11
    assert all(r.time.frames == recipes[0].preview.frames for r in recipes)  # preview variants


def test_batched_instances_are_a_sweep_of_the_base_recipe():
    """The batched runs' instances come from the sweep front-end: the base recipe with each instance's
    overrides applied, checked like any recipe, in order."""
    from plume_b200.recipe.derived import derive
    from plume_b200.recipe.variation import sweep_table
    from plume_b200.workloads import BATCH_GRIDS, batch_base_table, batch_variations, batched_recipes

    variations = batch_variations(count=5, seed=3)
    recipes = batched_recipes(count=5, frames=6, seed=3)
    assert [r.seed for r in recipes] == [7 + n for n in range(5)]
    for recipe, sets in zip(recipes, variations):
        values = dict(item.split("=", 1) for item in sets)
        assert derive(recipe).cells in BATCH_GRIDS
        assert recipe.domain.cell_m == float(values["domain.cell_m"])
        assert recipe.emitter[0].radius_m == float(values["emitter.puff.radius_m"])
        assert recipe.forces.drag_per_s == float(values["forces.drag_per_s"])
        assert recipe.time.frames == 6
    assert sweep_table(batch_base_table(6), variations, "batch") == recipes
