"""The recipe error type (mirrors chadmv/plume src/plume/recipe/errors.py:4-5)."""


class RecipeError(Exception):
    """A problem with a recipe's values, raised on the host before or between device work."""
