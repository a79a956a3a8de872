"""The slice plane's device steps (mirrors chadmv/plume src/plume/view/slice_plane.py:104-137 and the fields
it shows): cell-centre velocity, its curl (swirl), speed, and the plane coloured over the volume's display
bytes with the rest dimmed."""

import numpy as np
import torch

from plume_b200 import _native as N

DIM = 0.4
RAMP_STOPS = ((0.0, (0.07, 0.04, 0.33)), (0.25, (0.17, 0.33, 0.55)), (0.5, (0.13, 0.57, 0.55)),
              (0.75, (0.37, 0.79, 0.38)), (1.0, (0.99, 0.91, 0.15)))
RAMP_TABLE_SIZE = 256


def ramp_colors(count: int) -> np.ndarray:
    positions = np.linspace(0.0, 1.0, count)
    stops = np.array([stop for stop, _ in RAMP_STOPS])
    colors = np.array([color for _, color in RAMP_STOPS])
    return np.stack([np.interp(positions, stops, colors[:, channel]) for channel in range(3)], axis=-1)


def center_velocity(grid) -> torch.Tensor:
    """(nx, ny, nz, 3) cell-centre velocity of the grid's faces."""
    out = torch.empty((*grid.cells, 3), dtype=torch.float32, device=grid.device)
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_view_center_velocity", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(out), N.stream())
    return out


def curl(info, centers: torch.Tensor) -> torch.Tensor:
    out = torch.empty_like(centers)
    N.call("plume_view_curl", info, N.ptr(centers), N.ptr(out), N.stream())
    return out


def speed(vectors: torch.Tensor) -> torch.Tensor:
    out = torch.empty(vectors.shape[:-1], dtype=torch.float32, device=vectors.device)
    N.call("plume_view_speed", N.ptr(vectors), out.numel(), N.ptr(out), N.stream())
    return out


class SliceDrawer:
    def __init__(self, device: str):
        self.ramp = torch.from_numpy(ramp_colors(RAMP_TABLE_SIZE).astype(np.float32)).to(device)

    def overlay(self, image: torch.Tensor, view, info, axis: int, coordinate_m: float, values: torch.Tensor,
                low: float, high: float) -> None:
        """Draws `values` on the plane axis = coordinate_m over the display bytes `image` (in place)."""
        N.call("plume_view_slice", view, info, axis, coordinate_m, N.ptr(values), low, high, N.ptr(self.ramp),
               self.ramp.shape[0], N.ptr(image, torch.uint8), image.shape[0], image.shape[1], N.stream())


def field_range(values: np.ndarray, temperature: bool) -> tuple[float, float]:
    high = float(values.max()) if values.size else 1.0
    low = float(values.min()) if temperature and values.size else 0.0
    if not high > low:
        high = low + 1.0
    return low, high
