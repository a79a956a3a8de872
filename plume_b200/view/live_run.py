"""The live run's device helpers (mirrors chadmv/plume src/plume/view/live_run.py:42-72 and
view/frame_cache.py:26-50): the smoke's six boundary layers, the faces they show smoke on, and the frame
cache's float32 <-> float16 casts."""

import math

import numpy as np
import torch

from plume_b200 import _native as N

FACE_NAMES = ("left", "right", "bottom", "top", "back", "front")
CEILING = "top"


def boundary_layers(smoke: torch.Tensor) -> torch.Tensor:
    """(6, S, S) with S the largest dimension: layers[face, a, b], a and b the face's other axes in x, y, z
    order, 0 past the face's size."""
    side = max(smoke.shape)
    layers = torch.empty((6, side, side), dtype=torch.float32, device=smoke.device)
    N.call("plume_view_boundary_layers", N.ptr(smoke), N.shape3(smoke), N.ptr(layers), N.stream())
    return layers


def visible_density(recipe) -> float:
    return -math.log(1.0 - 1.0 / 255.0) / (recipe.render.opacity_per_density * recipe.domain.cell_m)


def faces_reached(layers: np.ndarray, recipe) -> tuple:
    largest = layers.reshape(len(FACE_NAMES), -1).max(axis=1)
    threshold = visible_density(recipe)
    faces = recipe.domain.faces
    return tuple(name for name, value in zip(FACE_NAMES, largest, strict=True)
                 if value >= threshold and (name == CEILING or getattr(faces, name) == "open"))


def narrow(source: torch.Tensor) -> torch.Tensor:
    """float32 -> float16 on the device (the frame cache's kept copy)."""
    out = torch.empty(source.shape, dtype=torch.float16, device=source.device)
    N.call("plume_view_narrow", N.ptr(source), N.ptr(out, torch.float16), source.numel(), N.stream())
    return out


def widen(source: torch.Tensor) -> torch.Tensor:
    out = torch.empty(source.shape, dtype=torch.float32, device=source.device)
    N.call("plume_view_widen", N.ptr(source, torch.float16), N.ptr(out), source.numel(), N.stream())
    return out
