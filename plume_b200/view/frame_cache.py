"""The viewer's frame cache (mirrors chadmv/plume src/plume/view/frame_cache.py:52-183): each kept frame's smoke
and temperature, and its velocity at cell centres, as float16 on the device, within a byte budget. The plan
keeps every frame with velocity when that fits; else every frame without velocity; else every second, fourth,
... frame without velocity. Reads widen a kept frame into the reader's own float32 scratch."""

import math

import torch

from plume_b200 import _native as N
from plume_b200.sim.grid import make_info

SCALAR_FIELDS = 2
VELOCITY_VALUES = 3
BYTES_PER_VALUE = 2


def narrow(source: torch.Tensor) -> torch.Tensor:
    """float32 -> float16 on the device (frame_cache.py:26-29, the kept copy); any shape."""
    out = torch.empty(source.shape, dtype=torch.float16, device=source.device)
    N.call("plume_view_narrow", N.ptr(source.contiguous()), N.ptr(out, torch.float16), source.numel(), N.stream())
    return out


def widen(source: torch.Tensor) -> torch.Tensor:
    """float16 -> float32 on the device (frame_cache.py:32-35)."""
    out = torch.empty(source.shape, dtype=torch.float32, device=source.device)
    N.call("plume_view_widen", N.ptr(source.contiguous(), torch.float16), N.ptr(out), source.numel(), N.stream())
    return out


def frame_bytes(cells, velocity: bool = False) -> int:
    return (SCALAR_FIELDS + (VELOCITY_VALUES if velocity else 0)) * BYTES_PER_VALUE * math.prod(cells)


def frame_stride(frames: int, cells, budget_bytes: float) -> int:
    """The smallest power-of-two stride whose kept frames fit the budget without velocity (at least one)."""
    stride = 1
    while stride < frames and math.ceil(frames / stride) * frame_bytes(cells) > budget_bytes:
        stride *= 2
    return stride


def keeps_velocity(frames: int, cells, budget_bytes: float) -> bool:
    return frames * frame_bytes(cells, velocity=True) <= budget_bytes


def _ordinal(number: int) -> str:
    suffix = {1: "st", 2: "nd", 3: "rd"}.get(number % 10 if number % 100 not in (11, 12, 13) else 0, "th")
    return f"{number}{suffix}"


class FrameCache:
    """Kept frames of one run, filled in frame order as the run lands them."""

    def __init__(self, cells, frames: int, budget_bytes: float, device: str, shared_with_compare: bool = False):
        self.cells = tuple(cells)
        self.frames = frames
        self.budget_bytes = budget_bytes
        self.device = device
        self.shared_with_compare = shared_with_compare
        self.has_velocity = keeps_velocity(frames, self.cells, budget_bytes)
        self.stride = 1 if self.has_velocity else frame_stride(frames, self.cells, budget_bytes)
        self._stored = {}
        self._velocity = {}
        self._centred = None
        self._info = make_info(self.cells, 1.0, (0.0, 0.0, 0.0), (0, 0, 0), (0, 0, 0))  # dimensions only

    def keeps(self, frame: int) -> bool:
        return frame % self.stride == 0

    def store(self, frame: int, smoke: torch.Tensor, temperature: torch.Tensor, velocity=None) -> None:
        """Rounds a kept frame's fields to float16 and keeps them; `velocity` (u, v, w face arrays) is kept at
        cell centres when the plan keeps velocity. Frames off the stride are ignored."""
        if not self.keeps(frame):
            return
        self._stored[frame] = (narrow(smoke.contiguous()), narrow(temperature.contiguous()))
        if self.has_velocity and velocity is not None:
            if self._centred is None:
                self._centred = torch.empty((*self.cells, 3), dtype=torch.float32, device=self.device)
            u, v, w = velocity
            N.call("plume_view_center_velocity", self._info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(self._centred),
                   N.stream())
            self._velocity[frame] = narrow(self._centred)

    def kept_frames(self) -> list:
        return sorted(self._stored)

    def nearest_kept(self, frame: int):
        kept = self.kept_frames()
        if not kept:
            return None
        earlier = [index for index in kept if index <= frame]
        return earlier[-1] if earlier else kept[0]

    @property
    def stored_bytes(self) -> int:
        return (len(self._stored) * frame_bytes(self.cells)
                + len(self._velocity) * (frame_bytes(self.cells, velocity=True) - frame_bytes(self.cells)))

    @property
    def thinned(self) -> bool:
        return self.stride > 1

    def scratch(self):
        return (torch.zeros(self.cells, dtype=torch.float32, device=self.device),
                torch.zeros(self.cells, dtype=torch.float32, device=self.device))

    def velocity_scratch(self) -> torch.Tensor:
        return torch.zeros((*self.cells, 3), dtype=torch.float32, device=self.device)

    def load(self, frame: int, into):
        """A kept frame's smoke and temperature widened to float32 into the reader's `into` pair."""
        for source, target in zip(self._stored[frame], into, strict=True):
            target.copy_(widen(source))
        return into

    def velocity_kept(self, frame: int) -> bool:
        return frame in self._velocity

    def load_velocity(self, frame: int, into: torch.Tensor) -> torch.Tensor:
        into.copy_(widen(self._velocity[frame]))
        return into

    def stored_smoke(self, frame: int) -> torch.Tensor:
        return self._stored[frame][0]

    def stored_velocity(self, frame: int) -> torch.Tensor:
        return self._velocity[frame]

    def thinning_note(self):
        """A status line when the budget made the cache drop velocity or skip frames, else None."""
        if self.has_velocity:
            return None
        gigabytes = self.budget_bytes / 2**30
        room = "the room the Compare run leaves of --cache-gb" if self.shared_with_compare else "--cache-gb"
        if self.stride == 1:
            return (f"frame cache keeps no velocity (the slice plane offers smoke and temperature only): "
                    f"{self.frames} frames at {frame_bytes(self.cells, velocity=True) / 2**20:.1f} MB each with "
                    f"velocity do not fit {gigabytes:.3g} GB ({room})")
        return (f"frame cache keeps every {_ordinal(self.stride)} frame and no velocity: {self.frames} frames at "
                f"{frame_bytes(self.cells) / 2**20:.1f} MB each do not fit {gigabytes:.3g} GB ({room})")
