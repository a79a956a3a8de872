"""Recipe loading (tests/recipe/test_load.py in chadmv/plume): defaults, derived grid and timing, the errors a
bad recipe gets (with the key path named), the preview rule. Host only."""

import pytest

from plume_b200.recipe.derived import derive
from plume_b200.recipe.errors import RecipeError
from plume_b200.recipe.load import load_recipe, preview_substeps

MINIMAL = """
[domain]
size_m = [2.0, 3.0, 2.0]
cell_m = 0.02

[time]
duration_s = 3.2

[[emitter]]
name = "puff"
center_m = [0.0, 0.3, 0.0]
radius_m = 0.25
end_s = 0.25
"""


def write(tmp_path, text, name="puff_test.toml"):
    path = tmp_path / name
    path.write_text(text)
    return path


def test_a_minimal_recipe_fills_the_defaults(tmp_path):
    recipe = load_recipe(write(tmp_path, MINIMAL))
    assert recipe.time.frames == 64 and recipe.output.columns == 8 and recipe.output.name == "puff_test"
    assert recipe.camera.seat == "puff" and recipe.emitter[0].temperature_k == 293.0
    assert recipe.domain.faces.bottom == "closed" and recipe.domain.faces.top == "open"


def test_the_derived_grid_and_timing(tmp_path):
    derived = derive(load_recipe(write(tmp_path, MINIMAL)))
    assert derived.cells == (100, 150, 100)
    assert derived.fps == pytest.approx(20.0) and derived.dt_s == pytest.approx(1.0 / 60.0)
    assert derived.domain_min_m == pytest.approx((-1.0, 0.0, -1.0))


@pytest.mark.parametrize("text,message", [
    (MINIMAL.replace("radius_m", "radius_n"), r"emitter\[0\]\.radius_n; did you mean radius_m"),
    (MINIMAL.replace("size_m = [2.0, 3.0, 2.0]\n", ""), r"domain\.size_m is required"),
    (MINIMAL.replace("duration_s = 3.2", 'duration_s = "long"'), r"time\.duration_s must be a number"),
    (MINIMAL + '\n[domain.faces]\ntop = "shut"\n', r"domain\.faces\.top must be one of closed, open"),
    (MINIMAL.replace("[[emitter]]", "[emitter]"), r"\[\[emitter\]\]"),
    (MINIMAL + '\n[camera]\nseat = "nowhere"\n', r"camera\.seat 'nowhere' is not an emitter"),
], ids=["typo", "missing", "type", "choice", "single-emitter-table", "seat"])
def test_a_bad_recipe_names_what_is_wrong(tmp_path, text, message):
    with pytest.raises(RecipeError, match=message):
        load_recipe(write(tmp_path, text))


@pytest.mark.parametrize("name", ["../escape", "a/b", "..", "C:evil", " spaced"])
def test_the_output_name_must_be_a_plain_name(tmp_path, name):
    with pytest.raises(RecipeError, match=r"output\.name must be a plain name"):
        load_recipe(write(tmp_path, MINIMAL + f'\n[output]\nname = "{name}"\n'))


@pytest.mark.parametrize("value", ["nan", "inf", "-inf"])
def test_non_finite_numbers_are_rejected(tmp_path, value):
    with pytest.raises(RecipeError, match=r"time\.duration_s must be a finite number"):
        load_recipe(write(tmp_path, MINIMAL.replace("duration_s = 3.2", f"duration_s = {value}")))


def test_a_non_finite_number_in_a_list_is_rejected(tmp_path):
    with pytest.raises(RecipeError, match=r"emitter\[0\]\.center_m\[1\] must be a finite number"):
        load_recipe(write(tmp_path, MINIMAL.replace("center_m = [0.0, 0.3, 0.0]", "center_m = [0.0, nan, 0.0]")))


def test_a_whole_number_too_large_for_a_float_is_rejected(tmp_path):
    with pytest.raises(RecipeError, match=r"time\.duration_s must be a finite number, got inf$"):
        load_recipe(write(tmp_path, MINIMAL.replace("duration_s = 3.2", f"duration_s = {10**400}")))


@pytest.mark.parametrize("center", ["[1.3, 0.3, 0.0]", "[-1.3, 0.3, 0.0]", "[0.0, -0.3, 0.0]", "[0.0, 3.3, 0.0]",
                                    "[0.0, 0.3, 1.3]"])
def test_an_emitter_wholly_outside_the_domain_is_rejected(tmp_path, center):
    with pytest.raises(RecipeError, match=r"emitter\[0\] lies outside the domain on [xyz]"):
        load_recipe(write(tmp_path, MINIMAL.replace("center_m = [0.0, 0.3, 0.0]", f"center_m = {center}")))


def test_a_box_emitter_wholly_outside_the_domain_is_rejected(tmp_path):
    text = MINIMAL.replace("center_m = [0.0, 0.3, 0.0]\nradius_m = 0.25",
                           'shape = "box"\ncenter_m = [0.0, -0.3, 0.0]\nsize_m = [0.5, 0.5, 0.5]')
    with pytest.raises(RecipeError, match=r"emitter\[0\] lies outside the domain on y"):
        load_recipe(write(tmp_path, text))


@pytest.mark.parametrize("center", ["[0.0, -0.1, 0.0]", "[1.2, 0.3, -1.2]", "[0.0, -0.25, 0.0]"])
def test_an_emitter_centred_outside_but_reaching_in_is_accepted(tmp_path, center):
    path = write(tmp_path, MINIMAL.replace("center_m = [0.0, 0.3, 0.0]", f"center_m = {center}"))
    assert load_recipe(path).emitter[0].radius_m == 0.25


def test_a_duration_too_small_for_its_frames_is_rejected(tmp_path):
    with pytest.raises(RecipeError, match=r"time\.duration_s is too small"):
        load_recipe(write(tmp_path, MINIMAL.replace("duration_s = 3.2", "duration_s = 1e-320")))


@pytest.mark.parametrize("seed", [-1, 2**31, 5_000_000_000])
def test_a_seed_outside_32_bits_is_rejected(tmp_path, seed):
    with pytest.raises(RecipeError, match=r"seed must be between 0 and 2147483647"):
        load_recipe(write(tmp_path, f"seed = {seed}\n" + MINIMAL))


def test_the_largest_seed_is_accepted(tmp_path):
    assert load_recipe(write(tmp_path, f"seed = {2**31 - 1}\n" + MINIMAL)).seed == 2**31 - 1


def test_the_preview_coarsens_the_longest_axis_to_48_cells(tmp_path):
    recipe = load_recipe(write(tmp_path, MINIMAL), preview=True)
    derived = derive(recipe)
    assert max(derived.cells) == 48 and recipe.time.frames == 16
    assert recipe.output.frame_px == 128 and recipe.output.columns == 4 and derived.fps == pytest.approx(5.0)


def test_the_preview_keeps_the_full_runs_step_length(tmp_path):
    full = derive(load_recipe(write(tmp_path, MINIMAL)))
    preview = derive(load_recipe(write(tmp_path, MINIMAL), preview=True))
    assert preview.steps_per_frame == 12  # 64 frames x 3 substeps over 16 frames
    assert preview.dt_s == pytest.approx(full.dt_s) and preview.warmup_steps == full.warmup_steps


def test_preview_substeps_round_up():
    assert preview_substeps(frames=64, substeps=3, preview_frames=16) == 12
    assert preview_substeps(frames=50, substeps=3, preview_frames=16) == 10
    assert preview_substeps(frames=8, substeps=1, preview_frames=16) == 1


@pytest.mark.parametrize("name", ["puff.core", "puff[0]", ""])
def test_an_emitter_name_a_key_path_cannot_hold_is_rejected(tmp_path, name):
    with pytest.raises(RecipeError, match=r"emitter\[0\]\.name must be a name without"):
        load_recipe(write(tmp_path, MINIMAL.replace('name = "puff"', f'name = "{name}"')))
