"""Assembling the sheet's frames on the device (mirrors chadmv/plume src/plume/sheet/assemble.py:39-77 and
the steps it calls: crop.py, resample.py, soften.py, shade.py, quantize.py, pack.py).

Same order as the reference: content box over every frame, square crop with margin, bicubic resampling of the
padded crop, soften, (shade layout) ease thin pixels and the shade divisor, the heat divisor, quantise, and
the gutter check, growing the margin and starting over from the crop while content reaches a frame's edge.
Only the content box (4 integers), the divisors and the gutter flag come back to the host until the finished
8-bit frames are copied once at the end.
"""

import math
from dataclasses import dataclass

import numpy as np
import torch

from plume_b200 import _native as N
from plume_b200.recipe.schema import NORMAL_LAYOUT, SHADE_LAYOUT
from plume_b200.render.raw_frame import CHANNELS, HEAT, SHADE, THICKNESS, empty_pixel
from plume_b200.sheet.resample import identity, taps

GUTTER_PX = 2            # assemble.py:19
MARGIN_GROWTH = 0.02
MAX_MARGIN_TRIES = 8
PAD_SLACK_PX = 4         # resample.py:13


@dataclass(frozen=True)
class CropSquare:
    """A square in domain-view pixel coordinates (crop.py:13-23)."""

    left: float
    top: float
    side: float

    def box(self) -> tuple[float, float, float, float]:
        return (self.left, self.top, self.left + self.side, self.top + self.side)


class NothingVisibleError(Exception):
    """No frame shows any smoke or heat, so there is nothing to crop to."""


class GutterError(Exception):
    """Content still reaches a frame's edge after growing the margin the maximum number of times."""


@dataclass(frozen=True)
class AssembledFrames:
    frames: list  # (frame_px, frame_px, 4) uint8 numpy arrays
    crop: CropSquare
    margin: float
    frame_m: float
    seat: tuple[float, float]
    heat_divisor: float
    shade_divisor: float | None
    device_frames: torch.Tensor  # (frames, frame_px, frame_px, 4) uint8 on the device


def square_crop(box, margin: float) -> CropSquare:
    left, top, right, bottom = box
    side = max(right - left, bottom - top) * (1.0 + 2.0 * margin)
    center_x = (left + right) / 2.0
    center_y = (top + bottom) / 2.0
    return CropSquare(left=center_x - side / 2.0, top=center_y - side / 2.0, side=side)


def gaussian_weights(sigma: float) -> np.ndarray:
    radius = math.ceil(3.0 * sigma)
    offsets = np.arange(-radius, radius + 1, dtype=np.float64)
    weights = np.exp(-offsets**2 / (2.0 * sigma**2))
    return weights / weights.sum()


def as_device_frames(raw_frames, device: str) -> torch.Tensor:
    """(frames, height, width, 5) float32 on the device, from a tensor or a list of arrays/tensors."""
    if isinstance(raw_frames, torch.Tensor):
        stack = raw_frames
    else:
        stack = torch.stack([torch.as_tensor(np.asarray(f) if not isinstance(f, torch.Tensor) else f)
                             .to(device=device, dtype=torch.float32) for f in raw_frames])
    stack = stack.to(device=device, dtype=torch.float32).contiguous()
    if stack.ndim != 4 or stack.shape[3] != CHANNELS:
        raise ValueError(f"raw frames must be (frames, height, width, {CHANNELS}), not {tuple(stack.shape)}")
    return stack


class SheetAssembler:
    """Device buffers for assembling `frames` raw frames of (height, width) into frame_px squares."""

    def __init__(self, frames: int, frame_px: int, device: str):
        self.device = device
        self.frame_px = frame_px
        dbl = dict(dtype=torch.float64, device=device)
        self.frame = torch.empty((frames, frame_px, frame_px, CHANNELS), **dbl)
        self.blurred = torch.empty_like(self.frame)
        self.scratch = torch.empty_like(self.frame)
        self.sums = torch.empty(2 * frames, **dbl)
        self.rgba = torch.empty((frames, frame_px, frame_px, 4), dtype=torch.uint8, device=device)
        self.heat_key = torch.empty(1, dtype=torch.int32, device=device)
        self.box = torch.empty(4, dtype=torch.int32, device=device)
        self.max_key = torch.empty(1, dtype=torch.int64, device=device)
        self.any = torch.empty(1, dtype=torch.int32, device=device)
        self.max_out = torch.empty(2, **dbl)
        self.touched = torch.empty(1, dtype=torch.int32, device=device)

    def content_box(self, raw: torch.Tensor):
        f, h, w, _ = raw.shape
        N.call("plume_sheet_content_box", N.ptr(raw), f, h, w, N.ptr(self.heat_key, torch.int32),
               N.ptr(self.box, torch.int32), N.stream())
        left, top, right, bottom = (int(x) for x in self.box.cpu())
        if right <= left or bottom <= top:
            raise NothingVisibleError("no frame shows any smoke or heat; check the emitters and the camera")
        return left, top, right, bottom

    def resample(self, raw: torch.Tensor, crop: CropSquare, channels: str) -> None:
        """resample.py:16-41 into self.frame."""
        f, height, width, _ = raw.shape
        left, top, right, bottom = crop.box()
        overflow = max(0.0, -left, -top, right - width, bottom - height)
        pad = math.ceil(overflow) + PAD_SLACK_PX
        padded_w, padded_h = width + 2 * pad, height + 2 * pad
        x0, y0, x1, y1 = left + pad, top + pad, right + pad, bottom + pad
        out = self.frame_px
        bx0, by0, bx1, by1 = (np.float32(v) for v in (x0, y0, x1, y1))  # Pillow's float32 box
        need_h = out != padded_w or bx0 != 0 or bx1 != out
        need_v = out != padded_h or by0 != 0 or by1 != out
        vertical = taps(padded_h, y0, y1, out)
        row_first = int(vertical.first[0])
        row_last = int(vertical.first[-1] + vertical.count[-1])
        horizontal = taps(padded_w, x0, x1, out) if need_h else identity(out)
        vertical = type(vertical)(vertical.first - row_first, vertical.count, vertical.weights)
        if not need_v:
            vertical = identity(out)
        rows = row_last - row_first
        dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(self.device, dt)  # noqa: E731
        hf, hc, hw = dev(horizontal.first, torch.int32), dev(horizontal.count, torch.int32), dev(horizontal.weights, torch.float64)
        vf, vc, vw = dev(vertical.first, torch.int32), dev(vertical.count, torch.int32), dev(vertical.weights, torch.float64)
        temp = torch.empty((f, CHANNELS, rows, out), dtype=torch.float32, device=self.device)
        empty = (N.ctypes.c_float * CHANNELS)(*empty_pixel(channels).tolist())
        N.call("plume_sheet_resample", N.ptr(raw), f, height, width, pad, empty,
               N.ptr(hf, torch.int32), N.ptr(hc, torch.int32), N.ptr(hw, torch.float64), horizontal.ksize,
               N.ptr(vf, torch.int32), N.ptr(vc, torch.int32), N.ptr(vw, torch.float64), vertical.ksize,
               row_first, rows, out, 1 if channels == SHADE_LAYOUT else 0, N.ptr(temp), N.ptr(self.frame, torch.float64),
               N.stream())

    def blur(self, src: torch.Tensor, dst: torch.Tensor, sigma: float, offset: int, channels: int) -> None:
        weights = torch.from_numpy(gaussian_weights(sigma)).to(self.device)
        frames, size = src.shape[0], src.shape[1]
        N.call("plume_sheet_blur", N.ptr(src, torch.float64), N.ptr(dst, torch.float64),
               N.ptr(self.scratch, torch.float64), frames, size, channels, CHANNELS, offset,
               N.ptr(weights, torch.float64), (len(weights) - 1) // 2, N.stream())

    def channel_max(self, channel: int, floor: float) -> tuple[float, bool]:
        frames, size = self.frame.shape[0], self.frame.shape[1]
        N.call("plume_sheet_channel_max", N.ptr(self.frame, torch.float64), frames, size, channel, floor,
               N.ptr(self.max_key, torch.int64), N.ptr(self.any, torch.int32), N.ptr(self.max_out, torch.float64),
               N.stream())
        value, found = self.max_out.cpu().tolist()
        return value, found > 0.0

    def finish(self, render, channels: str) -> tuple[float, float | None]:
        """soften, ease and divisors (assemble.py:50-56) on self.frame; returns (heat, shade) divisors."""
        frames, size = self.frame.shape[0], self.frame.shape[1]
        if render.soften_px > 0.0:
            self.blur(self.frame, self.frame, render.soften_px, 0, CHANNELS)
        if channels == NORMAL_LAYOUT:
            N.call("plume_sheet_renormalize", N.ptr(self.frame, torch.float64), frames, size, N.stream())
        divisor = None
        if channels == SHADE_LAYOUT:
            if render.shade_neighborhood_px > 0.0:
                self.blur(self.frame, self.blurred, render.shade_neighborhood_px, THICKNESS, 2)
                blurred = self.blurred
            else:
                blurred = self.frame
            N.call("plume_sheet_ease", N.ptr(self.frame, torch.float64), N.ptr(blurred, torch.float64),
                   N.ptr(self.sums, torch.float64), frames, size, render.shade_fade_thickness, N.stream())
            divisor = 1.0
            for floor in (render.shade_fade_thickness, np.finfo(np.float64).tiny):  # shade.py:45-55
                largest, found = self.channel_max(SHADE, floor)
                if found and largest > 0.0:
                    divisor = largest
                    break
        heat_divisor, _ = self.channel_max(HEAT, -math.inf)
        return heat_divisor, divisor

    def quantize(self, heat_divisor: float, shade_divisor: float | None, channels: str) -> bool:
        """Quantises self.frame into self.rgba; True when the gutter is empty."""
        frames, size = self.frame.shape[0], self.frame.shape[1]
        N.call("plume_sheet_quantize", N.ptr(self.frame, torch.float64), frames, size, heat_divisor,
               shade_divisor or 1.0, 1 if channels == SHADE_LAYOUT else 0, GUTTER_PX, N.ptr(self.rgba, torch.uint8),
               N.ptr(self.touched, torch.int32), N.stream())
        return int(self.touched.item()) == 0


def assemble(raw_frames, view, seat_world_m, frame_px: int, render, channels: str,
             device: str = "cuda:0") -> AssembledFrames:
    """The quantised frames and the facts the JSON and reports need (assemble.py:39-60)."""
    raw = as_device_frames(raw_frames, device)
    work = SheetAssembler(raw.shape[0], frame_px, device)
    box = work.content_box(raw)
    margin = render.crop_margin
    for _ in range(MAX_MARGIN_TRIES + 1):
        crop = square_crop(box, margin)
        work.resample(raw, crop, channels)
        heat_divisor, divisor = work.finish(render, channels)
        if work.quantize(heat_divisor, divisor, channels):
            device_frames = work.rgba.clone()
            host = device_frames.cpu().numpy()
            x, y = view.to_pixels(np.asarray(seat_world_m, dtype=np.float64))
            return AssembledFrames(frames=[host[i] for i in range(host.shape[0])], crop=crop, margin=margin,
                                   frame_m=crop.side * view.pixel_m,
                                   seat=((x - crop.left) / crop.side, (y - crop.top) / crop.side),
                                   heat_divisor=heat_divisor, shade_divisor=divisor, device_frames=device_frames)
        margin += MARGIN_GROWTH
    raise GutterError(f"content still touches the frame edge with crop_margin {margin:.2f}")


def pack(frames: torch.Tensor, columns: int) -> torch.Tensor:
    """pack.py:13-20 on the device: (rows * size, columns * size, 4) uint8, slots past the last frame zero."""
    count, size = frames.shape[0], frames.shape[1]
    rows = math.ceil(count / columns)
    sheet = torch.empty((rows * size, columns * size, 4), dtype=torch.uint8, device=frames.device)
    N.call("plume_sheet_pack", N.ptr(frames.contiguous(), torch.uint8), count, size, columns,
           N.ptr(sheet, torch.uint8), N.stream())
    return sheet
