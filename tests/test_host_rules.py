"""Host-side rules of the reference's simulation tests (tests/sim/test_forces.py, test_conserve.py in
chadmv/plume) that need no device."""

import pytest

from support import tiny_recipe


def test_wind_without_drag_is_a_recipe_error():
    from plume_b200.recipe.errors import RecipeError

    with pytest.raises(RecipeError, match="drag_per_s"):
        tiny_recipe(forces={"wind_mps": [1.0, 0.0, 0.0]})


def test_held_total_removes_gains_and_keeps_the_plain_pass_floor():
    from plume_b200.sim.conserve import held_total

    assert held_total(before=10.0, semi_lagrangian=9.0, maccormack=12.0) == 10.0  # a gain is removed
    assert held_total(before=10.0, semi_lagrangian=9.0, maccormack=9.5) == 9.5  # within bounds: unchanged
    assert held_total(before=10.0, semi_lagrangian=9.0, maccormack=8.0) == 9.0  # never below the plain pass
    assert held_total(before=10.0, semi_lagrangian=4.0, maccormack=3.0) == 4.0  # outflow as the scheme has it
