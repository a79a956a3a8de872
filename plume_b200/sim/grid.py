"""The MAC grid state on the device (mirrors chadmv/plume src/plume/sim/grid.py:15-94).

Fields are torch tensors, C-contiguous, shape (nx, ny, nz) with z contiguous; face velocities are
(nx+1, ny, nz), (nx, ny+1, nz), (nx, ny, nz+1). Sample positions are `index + offset` in cell units.
Velocity, smoke and temperature are float32 as in the reference, or, for the mixed-precision step, bfloat16
or float16 storage (every kernel computes in float32); pressure and divergence are always float32.
"""

from dataclasses import dataclass

import torch

from plume_b200._native import PlumeGridInfo as GridInfo

CENTER = (0.5, 0.5, 0.5)
U_FACE = (0.0, 0.5, 0.5)
V_FACE = (0.5, 0.0, 0.5)
W_FACE = (0.5, 0.5, 0.0)


class AdvectedField:
    """One advected quantity: current values plus MacCormack's forward-pass (`hat`) and output (`next`)
    buffers. The backward pass is evaluated inside the correction kernel, so `back` is only allocated if a
    caller asks for it."""

    def __init__(self, shape, offset, outside: float, uses_outside: bool, device: str, initial: float = 0.0,
                 dtype=torch.float32):
        self.offset = offset
        self.outside = outside
        self.uses_outside = 1 if uses_outside else 0
        self.data = torch.full(shape, initial, dtype=dtype, device=device)
        self.hat = torch.zeros(shape, dtype=dtype, device=device)
        self.next = torch.zeros(shape, dtype=dtype, device=device)
        self._back = None

    @property
    def back(self) -> torch.Tensor:
        if self._back is None:
            self._back = torch.zeros_like(self.data)
        return self._back

    def swap(self) -> None:
        self.data, self.next = self.next, self.data


@dataclass
class Grid:
    info: GridInfo
    device: str
    cells: tuple
    u: AdvectedField
    v: AdvectedField
    w: AdvectedField
    smoke: AdvectedField
    temperature: AdvectedField
    pressure: torch.Tensor
    divergence: torch.Tensor

    def velocity_fields(self):
        return self.u, self.v, self.w

    @property
    def storage(self) -> torch.dtype:
        """The element type of the velocity, smoke and temperature arrays."""
        return self.smoke.data.dtype


def make_info(cells, cell_m, origin_m, open_lo, open_hi, fill_hi=(1.0, 1.0, 1.0), ghost_gap=0.5) -> GridInfo:
    info = GridInfo()
    info.dims = type(info.dims)(*cells)
    info.cell_m = cell_m
    info.origin_m = type(info.origin_m)(*origin_m)
    info.open_lo = type(info.open_lo)(*open_lo)
    info.open_hi = type(info.open_hi)(*open_hi)
    info.fill_hi = type(info.fill_hi)(*fill_hi)
    info.ghost_gap = ghost_gap
    return info


def _is_open(kind: str) -> int:
    return 1 if kind == "open" else 0


def make_grid(derived, cell_m: float, faces, ambient_k: float, device: str, storage=torch.float32) -> Grid:
    """Allocates a grid at rest, filled with ambient air; `storage` is the element type of the velocity, smoke
    and temperature arrays (float32, or bfloat16 / float16 for the mixed-precision step)."""
    if storage not in (torch.float32, torch.bfloat16, torch.float16):
        raise TypeError(f"storage must be float32, bfloat16 or float16, not {storage}")
    nx, ny, nz = derived.cells
    info = make_info(derived.cells, cell_m, derived.domain_min_m,
                     [_is_open(k) for k in (faces.left, faces.bottom, faces.back)],
                     [_is_open(k) for k in (faces.right, faces.top, faces.front)])
    cells = (nx, ny, nz)
    return Grid(info=info, device=device, cells=cells,
                u=AdvectedField((nx + 1, ny, nz), U_FACE, 0.0, False, device, dtype=storage),
                v=AdvectedField((nx, ny + 1, nz), V_FACE, 0.0, False, device, dtype=storage),
                w=AdvectedField((nx, ny, nz + 1), W_FACE, 0.0, False, device, dtype=storage),
                smoke=AdvectedField(cells, CENTER, 0.0, True, device, dtype=storage),
                temperature=AdvectedField(cells, CENTER, ambient_k, True, device, initial=ambient_k,
                                          dtype=storage),
                pressure=torch.zeros(cells, dtype=torch.float32, device=device),
                divergence=torch.zeros(cells, dtype=torch.float32, device=device))
