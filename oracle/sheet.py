"""CPU restatement of the reference's sheet assembly and numbers file, as the checker for the device sheet
path. Test infrastructure only: the product never imports this module.

Follows chadmv/plume src/plume/sheet/assemble.py:39-77, crop.py:29-50, resample.py:16-41, soften.py:12-53,
shade.py:22-55, quantize.py:20-39, pack.py:13-20 and src/plume/report/numbers.py:42-121. The reference
resamples with Pillow (a third-party dependency, Pillow 12.2 here) through Image.resize(BICUBIC, box) on 32-bit
float images; `resample_plane` restates that published algorithm (Pillow's two-pass separable convolution:
per output index a window of source indices and normalised bicubic weights, a = -0.5, the support widened by
the scale when shrinking; the horizontal pass over the rows the vertical pass needs, each pass accumulating
in double and storing float32) and is checked against Pillow itself in the tests.
"""

import math

import numpy as np

# raw frame channels (render/raw_frame.py:15-21)
HEAT, THICKNESS, SHADE, NORMAL_X, NORMAL_Y, NORMAL_Z = 0, 1, 2, 2, 3, 4
CHANNELS = 5
SHADE_LAYOUT = "heat,thickness,shade,unused"
NORMAL_LAYOUT = "heat,thickness,normal_x,normal_y"

CONTENT_LEVEL = 0.5 / 255.0        # crop.py:10
PAD_SLACK_PX = 4                   # resample.py:13
GUTTER_PX, MARGIN_GROWTH, MAX_MARGIN_TRIES = 2, 0.02, 8   # assemble.py:19-21
FRAME_MEAN_WEIGHT, NO_SMOKE = 1.0 / 255.0, 1e-12          # shade.py:17-20
FACING_BYTE, UNUSED_BYTE = 128, 255                        # quantize.py:17-18
COVERED_LEVEL, FADE_FRACTION = 8, 0.1                      # numbers.py:10-11


def empty_pixel(channels: str) -> np.ndarray:
    pixel = np.zeros(CHANNELS, dtype=np.float32)
    if channels == NORMAL_LAYOUT:
        pixel[NORMAL_Z] = 1.0
    return pixel


# ---- crop (crop.py:29-50) --------------------------------------------------------------------------------
def content_box(raw_frames):
    heat_max = max(float(frame[..., HEAT].max()) for frame in raw_frames)
    union = np.zeros(raw_frames[0].shape[:2], dtype=bool)
    for frame in raw_frames:
        union |= frame[..., THICKNESS] >= CONTENT_LEVEL
        if heat_max > 0.0:
            union |= frame[..., HEAT] >= CONTENT_LEVEL * heat_max
    rows = np.nonzero(union.any(axis=1))[0]
    columns = np.nonzero(union.any(axis=0))[0]
    if rows.size == 0:
        raise ValueError("no frame shows any smoke or heat")
    return int(columns[0]), int(rows[0]), int(columns[-1]) + 1, int(rows[-1]) + 1


def square_crop(box, margin: float):
    left, top, right, bottom = box
    side = max(right - left, bottom - top) * (1.0 + 2.0 * margin)
    center_x = (left + right) / 2.0
    center_y = (top + bottom) / 2.0
    return (center_x - side / 2.0, center_y - side / 2.0, side)


# ---- bicubic resampling of a float image (Pillow's algorithm) -----------------------------------------------
def _bicubic(x: float) -> float:
    a = -0.5
    x = abs(x)
    if x < 1.0:
        return ((a + 2.0) * x - (a + 3.0)) * x * x + 1
    if x < 2.0:
        return (((x - 5) * x + 8) * x - 4) * a
    return 0.0


def coefficients(in_size: int, in0: float, in1: float, out_size: int):
    """Per output index: the first source index, the window length and the normalised weights. Pillow takes
    the box as float32: the box edges and their difference are float32, the rest double."""
    in0, in1 = np.float32(in0), np.float32(in1)
    scale = filterscale = float(np.float32(in1 - in0)) / out_size
    in0 = float(in0)
    if filterscale < 1.0:
        filterscale = 1.0
    support = 2.0 * filterscale
    ksize = int(math.ceil(support)) * 2 + 1
    first = np.zeros(out_size, dtype=np.int64)
    count = np.zeros(out_size, dtype=np.int64)
    weights = np.zeros((out_size, ksize), dtype=np.float64)
    for xx in range(out_size):
        center = in0 + (xx + 0.5) * scale
        ss = 1.0 / filterscale
        xmin = int(center - support + 0.5)
        if xmin < 0:
            xmin = 0
        xmax = int(center + support + 0.5)
        if xmax > in_size:
            xmax = in_size
        xmax -= xmin
        total = 0.0
        for x in range(xmax):
            w = _bicubic((x + xmin - center + 0.5) * ss)
            weights[xx, x] = w
            total += w
        if total != 0.0:
            for x in range(xmax):
                weights[xx, x] /= total
        first[xx], count[xx] = xmin, xmax
    return first, count, weights


def resample_plane(plane: np.ndarray, box, out_size: int) -> np.ndarray:
    """Image.fromarray(plane float32).resize((out, out), BICUBIC, box=box) restated."""
    height, width = plane.shape
    x0, y0, x1, y1 = box
    hf, hc, hw = coefficients(width, x0, x1, out_size)
    vf, vc, vw = coefficients(height, y0, y1, out_size)
    row_first = int(vf[0])
    row_last = int(vf[-1] + vc[-1])
    src = plane.astype(np.float32)
    need_h = out_size != width or x0 != 0 or x1 != out_size
    need_v = out_size != height or y0 != 0 or y1 != out_size
    if need_h:
        temp = np.zeros((row_last - row_first, out_size), dtype=np.float32)
        for xx in range(out_size):
            f, c = int(hf[xx]), int(hc[xx])
            acc = np.zeros(row_last - row_first, dtype=np.float64)
            for x in range(c):
                acc = acc + src[row_first:row_last, f + x].astype(np.float64) * hw[xx, x]
            temp[:, xx] = acc.astype(np.float32)
        src = temp
        vf = vf - row_first
    if not need_v:
        return src
    out = np.zeros((out_size, src.shape[1]), dtype=np.float32)
    for yy in range(out_size):
        f, c = int(vf[yy]), int(vc[yy])
        acc = np.zeros(src.shape[1], dtype=np.float64)
        for y in range(c):
            acc = acc + src[f + y, :].astype(np.float64) * vw[yy, y]
        out[yy, :] = acc.astype(np.float32)
    return out


def pad_to_cover(raw, crop, channels):
    height, width = raw.shape[:2]
    left, top, side = crop
    right, bottom = left + side, top + side
    overflow = max(0.0, -left, -top, right - width, bottom - height)
    pad = math.ceil(overflow) + PAD_SLACK_PX
    padded = np.tile(empty_pixel(channels), (height + 2 * pad, width + 2 * pad, 1))
    padded[pad:pad + height, pad:pad + width] = raw
    return padded, pad


def resample_frame(raw, crop, frame_px, channels):
    padded, shift = pad_to_cover(raw, crop, channels)
    left, top, side = crop
    box = (left + shift, top + shift, left + side + shift, top + side + shift)
    planes = [resample_plane(padded[..., c], box, frame_px) for c in range(CHANNELS)]
    frame = np.stack(planes, axis=-1).astype(np.float64)
    frame[..., THICKNESS] = np.clip(frame[..., THICKNESS], 0.0, 1.0)
    frame[..., HEAT] = np.maximum(frame[..., HEAT], 0.0)
    if channels == SHADE_LAYOUT:
        frame[..., SHADE] = np.clip(frame[..., SHADE], 0.0, frame[..., THICKNESS])
    return frame


# ---- soften, shade, quantize (soften.py, shade.py, quantize.py) -------------------------------------------
def gaussian(sigma: float) -> np.ndarray:
    radius = math.ceil(3.0 * sigma)
    offsets = np.arange(-radius, radius + 1, dtype=np.float64)
    weights = np.exp(-offsets**2 / (2.0 * sigma**2))
    return weights / weights.sum()


def blur_axis(image, weights, axis):
    radius = len(weights) // 2
    pad = [(0, 0)] * image.ndim
    pad[axis] = (radius, radius)
    padded = np.pad(image, pad, mode="edge")
    size = image.shape[axis]
    result = np.zeros_like(image)
    for offset, weight in enumerate(weights):
        result += weight * np.take(padded, np.arange(offset, offset + size), axis=axis)
    return result


def blur(image, sigma):
    if sigma <= 0.0:
        return image
    weights = gaussian(sigma)
    return blur_axis(blur_axis(image, weights, 0), weights, 1)


def renormalize(frame):
    result = frame.copy()
    normal = result[..., NORMAL_X:NORMAL_Z + 1]
    normal[..., 2] = np.abs(normal[..., 2])
    length = np.linalg.norm(normal, axis=-1, keepdims=True)
    facing = np.array([0.0, 0.0, 1.0])
    result[..., NORMAL_X:NORMAL_Z + 1] = np.where(length > 1e-6, normal / np.maximum(length, 1e-6), facing)
    return result


def soften(frame, sigma, channels):
    result = blur(frame, sigma)
    return renormalize(result) if channels == NORMAL_LAYOUT else result


def ease_thin_pixels(frame, fade_thickness, neighborhood_px):
    thickness = frame[..., THICKNESS]
    weighted = frame[..., SHADE]
    total = float(thickness.sum())
    mean = float(weighted.sum()) / total if total > 0.0 else 0.0
    neighborhood = ((blur(weighted, neighborhood_px) + FRAME_MEAN_WEIGHT * mean)
                    / (blur(thickness, neighborhood_px) + FRAME_MEAN_WEIGHT))
    has_smoke = thickness > NO_SMOKE
    own = np.clip(np.where(has_smoke, weighted / np.where(has_smoke, thickness, 1.0), 0.0), 0.0, 1.0)
    weight = np.clip(thickness / fade_thickness, 0.0, 1.0)
    result = frame.copy()
    result[..., SHADE] = neighborhood + weight * (own - neighborhood)
    return result


def shade_divisor(frames, fade_thickness):
    for floor in (fade_thickness, np.finfo(np.float64).tiny):
        shades = [frame[..., SHADE][frame[..., THICKNESS] >= floor] for frame in frames]
        largest = max((float(v.max()) for v in shades if v.size), default=0.0)
        if largest > 0.0:
            return largest
    return 1.0


def to_byte(values):
    return np.clip(np.floor(values * 255.0 + 0.5), 0, 255).astype(np.uint8)


def quantize(frame, heat_divisor, channels, shade_div=1.0):
    heat = frame[..., HEAT] / heat_divisor if heat_divisor > 0.0 else np.zeros(frame.shape[:2])
    red_green = [to_byte(heat), to_byte(frame[..., THICKNESS])]
    if channels == SHADE_LAYOUT:
        return np.stack([*red_green, to_byte(frame[..., SHADE] / shade_div),
                         np.full(frame.shape[:2], UNUSED_BYTE, dtype=np.uint8)], axis=-1)
    rgba = np.stack([*red_green, to_byte((frame[..., NORMAL_X] + 1.0) * 0.5),
                     to_byte((frame[..., NORMAL_Y] + 1.0) * 0.5)], axis=-1)
    empty = (rgba[..., 0] == 0) & (rgba[..., 1] == 0)
    rgba[empty, 2] = FACING_BYTE
    rgba[empty, 3] = FACING_BYTE
    return rgba


def gutter_is_empty(frame):
    ring = np.ones(frame.shape[:2], dtype=bool)
    ring[GUTTER_PX:-GUTTER_PX, GUTTER_PX:-GUTTER_PX] = False
    return not np.any(frame[ring][:, :2])


def assemble(raw_frames, frame_px, render, channels):
    """(quantized frames, crop, margin, heat divisor, shade divisor) as assemble.py:39-60 finds them."""
    box = content_box(raw_frames)
    margin = render.crop_margin
    for _ in range(MAX_MARGIN_TRIES + 1):
        crop = square_crop(box, margin)
        finished = [soften(resample_frame(raw, crop, frame_px, channels), render.soften_px, channels)
                    for raw in raw_frames]
        divisor = None
        if channels == SHADE_LAYOUT:
            finished = [ease_thin_pixels(f, render.shade_fade_thickness, render.shade_neighborhood_px)
                        for f in finished]
            divisor = shade_divisor(finished, render.shade_fade_thickness)
        heat_divisor = max(float(f[..., HEAT].max()) for f in finished)
        frames = [quantize(f, heat_divisor, channels, divisor or 1.0) for f in finished]
        if all(gutter_is_empty(f) for f in frames):
            return frames, crop, margin, heat_divisor, divisor
        margin += MARGIN_GROWTH
    raise ValueError("content still touches the frame edge")


def pack(frames, columns):
    size = frames[0].shape[0]
    rows = math.ceil(len(frames) / columns)
    sheet = np.zeros((rows * size, columns * size, frames[0].shape[2]), dtype=frames[0].dtype)
    for index, frame in enumerate(frames):
        row, column = divmod(index, columns)
        sheet[row * size:(row + 1) * size, column * size:(column + 1) * size] = frame
    return sheet


# ---- numbers (report/numbers.py:42-77) ---------------------------------------------------------------------
def measure_frame(frame):
    """(coverage, box or None, mean_heat, mean_thick, total_thick, peak_heat) of one quantized frame."""
    heat = frame[..., 0].astype(np.float64) / 255.0
    thickness = frame[..., 1].astype(np.float64) / 255.0
    covered = frame[..., 1] >= COVERED_LEVEL
    size = frame.shape[0]
    box = None
    if covered.any():
        rows = np.nonzero(covered.any(axis=1))[0]
        columns = np.nonzero(covered.any(axis=0))[0]
        box = (columns[0] / size, rows[0] / size, (columns[-1] + 1) / size, (rows[-1] + 1) / size)
    return (float(covered.mean()), box, float(heat[covered].mean()) if covered.any() else 0.0,
            float(thickness[covered].mean()) if covered.any() else 0.0, float(thickness.sum()), float(heat.max()))
