"""The orthographic sheet camera and the domain view (host math, numpy float64).

Same conventions as chadmv/plume src/plume/render/camera.py:16-78: camera space is x right, y up, z toward the
camera; elevation looks down, azimuth orbits counter-clockwise seen from above starting on the +z side; the
domain view is the smallest pixel grid at `px_per_cell` covering the projected domain box, pixel (0, 0) at the
top left.
"""

import math
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Camera:
    right: np.ndarray
    up: np.ndarray
    toward: np.ndarray  # from the scene toward the camera (camera-space +z)

    def to_camera_space(self, world_vector: np.ndarray) -> np.ndarray:
        return np.array([world_vector @ self.right, world_vector @ self.up, world_vector @ self.toward])


def make_camera(elevation_deg: float, azimuth_deg: float) -> Camera:
    el, az = math.radians(elevation_deg), math.radians(azimuth_deg)
    toward = np.array([math.sin(az) * math.cos(el), math.sin(el), math.cos(az) * math.cos(el)])
    right = np.array([math.cos(az), 0.0, -math.sin(az)])
    up = np.cross(toward, right)
    return Camera(right=right, up=up / np.linalg.norm(up), toward=toward)


@dataclass(frozen=True)
class DomainView:
    camera: Camera
    left_m: float
    top_m: float
    pixel_m: float
    width_px: int
    height_px: int

    def to_pixels(self, world_point: np.ndarray) -> tuple[float, float]:
        x = (world_point @ self.camera.right - self.left_m) / self.pixel_m
        y = (self.top_m - world_point @ self.camera.up) / self.pixel_m
        return float(x), float(y)


def make_domain_view(camera: Camera, domain_min_m, domain_size_m, cell_m: float, px_per_cell: float) -> DomainView:
    low, size = np.array(domain_min_m), np.array(domain_size_m)
    corners = [low + size * np.array([a, b, c]) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
    xs = [corner @ camera.right for corner in corners]
    ys = [corner @ camera.up for corner in corners]
    pixel_m = cell_m / px_per_cell
    return DomainView(camera=camera, left_m=min(xs), top_m=max(ys), pixel_m=pixel_m,
                      width_px=math.ceil((max(xs) - min(xs)) / pixel_m - 1e-6),
                      height_px=math.ceil((max(ys) - min(ys)) / pixel_m - 1e-6))


def sheet_domain_view(recipe, derived) -> DomainView:
    camera = make_camera(recipe.camera.elevation_deg, recipe.camera.azimuth_deg)
    return make_domain_view(camera, derived.domain_min_m, derived.size_m, recipe.domain.cell_m,
                            recipe.render.px_per_cell)
