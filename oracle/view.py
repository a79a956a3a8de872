"""CPU restatement of the live viewer's device compute, as the checker for plume_b200's view kernels. Test
infrastructure only: the product never imports this module.

Follows chadmv/plume src/plume/view/viewport.py:62-140 (look_kernel, table_lookup, to_byte, srgb_byte,
center_depth_kernel), view/slice_plane.py:104-137 (speed_kernel, slice_kernel), sim/vorticity.py:17-45
(center_velocity_kernel, curl_kernel), view/live_run.py:42-57 (boundary_layer_kernel), render/raymarch.py:55-83
(slab_range, pixel_ray) and report/composite.py:55-67 (the host composite the look must match within a byte).
Float32 arithmetic in the reference's order, as numpy float32 arrays (no operation is fused).
"""

import numpy as np

F = np.float32
NO_SMOKE = F(1e-12)


def table_lookup(table: np.ndarray, value: np.ndarray) -> np.ndarray:
    n = table.shape[0]
    position = np.clip(value.astype(F), F(0.0), F(1.0)) * F(n - 1)
    low = np.minimum(position.astype(np.int32), n - 2)
    t = (position - low.astype(F))[..., None]
    return table[low] * (F(1.0) - t) + table[low + 1] * t


def to_byte(value: np.ndarray) -> np.ndarray:
    return np.clip(np.floor(value * F(255.0) + F(0.5)), F(0.0), F(255.0)).astype(np.int32).astype(np.uint8)


def srgb_byte(table: np.ndarray, linear: np.ndarray) -> np.ndarray:
    return table[(np.clip(linear, F(0.0), F(1.0)) * F(table.shape[0] - 1) + F(0.5)).astype(np.int32)]


def look(raw, smoke_ramp, emission_ramp, srgb, view, shade_layout, heat_divisor, shade_divisor, shade_depth,
         ambient, toward_light, background) -> np.ndarray:
    raw = raw.astype(F)
    heat = np.clip(raw[..., 0] / F(heat_divisor), F(0.0), F(1.0))
    thickness = np.clip(raw[..., 1], F(0.0), F(1.0))
    normal = raw[..., 2:5]
    shade = np.zeros_like(heat)
    if shade_layout:
        smoky = thickness > NO_SMOKE
        safe = np.where(smoky, thickness, F(1.0))
        shade = np.where(smoky, np.clip(raw[..., 2] / safe / F(shade_divisor), F(0.0), F(1.0)), F(0.0))
        light = F(1.0) - F(shade_depth) * (F(1.0) - shade)
    else:
        tl = np.asarray(toward_light, dtype=F)
        dot = (normal[..., 0] * tl[0] + normal[..., 1] * tl[1]) + normal[..., 2] * tl[2]
        light = F(ambient) + (F(1.0) - F(ambient)) * np.maximum(F(0.0), dot)
    out = np.zeros((*raw.shape[:2], 4), dtype=np.uint8)
    if view == 0:
        smoke = table_lookup(smoke_ramp, heat) * light[..., None]
        glow = table_lookup(emission_ramp, heat)
        bg = np.asarray(background, dtype=F)
        linear = (bg * (F(1.0) - thickness[..., None]) + smoke * thickness[..., None]) + glow
        out[..., :3] = srgb_byte(srgb, linear)
    else:
        gray = heat if view == 1 else (thickness if view == 2 else shade)
        color = np.repeat(gray[..., None], 3, axis=-1)
        if view == 3 and not shade_layout:
            color = (normal + F(1.0)) * F(0.5)
        out[..., :3] = to_byte(color)
    out[..., 3] = 255
    return out


def composite(rgba, background_linear, channels_shade: bool, look_settings, light_dir, ramp) -> np.ndarray:
    """report/composite.py:55-67 (float64): the frame over a flat background as linear RGB."""
    values = rgba.astype(np.float64) / 255.0
    heat, thickness = values[..., 0], values[..., 1]
    if channels_shade:
        light = 1.0 - look_settings.shade_depth * (1.0 - values[..., 2])
    else:
        nx = values[..., 2] * 2.0 - 1.0
        ny = values[..., 3] * 2.0 - 1.0
        nz = np.sqrt(np.maximum(0.0, 1.0 - nx**2 - ny**2))
        normal = np.stack([nx, ny, nz], axis=-1)
        toward = np.array(light_dir, dtype=np.float64)
        toward /= np.linalg.norm(toward)
        light = look_settings.ambient + (1.0 - look_settings.ambient) * np.maximum(0.0, normal @ toward)
    smoke = ramp(look_settings.smoke_ramp, heat) * light[..., None]
    glow = ramp(look_settings.emission_ramp, heat)
    return background_linear * (1.0 - thickness[..., None]) + thickness[..., None] * smoke + glow


# ---- sampling and rays -------------------------------------------------------------------------------------
def sample(field: np.ndarray, g) -> np.float32:
    """sample_index_space (sim/sample.py:10-29) at one point, float32."""
    n = field.shape
    x = [min(max(F(g[a]), F(0.0)), F(n[a] - 1)) for a in range(3)]
    i0 = [int(x[a]) for a in range(3)]
    i1 = [min(i0[a] + 1, n[a] - 1) for a in range(3)]
    t = [x[a] - F(i0[a]) for a in range(3)]
    lerp = lambda a, b, s: a * (F(1.0) - s) + b * s  # noqa: E731
    f = field.astype(F)
    c00 = lerp(f[i0[0], i0[1], i0[2]], f[i1[0], i0[1], i0[2]], t[0])
    c10 = lerp(f[i0[0], i1[1], i0[2]], f[i1[0], i1[1], i0[2]], t[0])
    c01 = lerp(f[i0[0], i0[1], i1[2]], f[i1[0], i0[1], i1[2]], t[0])
    c11 = lerp(f[i0[0], i1[1], i1[2]], f[i1[0], i1[1], i1[2]], t[0])
    return lerp(lerp(c00, c10, t[1]), lerp(c01, c11, t[1]), t[2])


def slab_range(origin, direction, bmin, bmax):
    t_enter, t_exit = F(-1.0e30), F(1.0e30)
    for a in range(3):
        if abs(direction[a]) < F(1.0e-12):
            if origin[a] < bmin[a] or origin[a] > bmax[a]:
                return F(1.0), F(0.0)
        else:
            t0 = (bmin[a] - origin[a]) / direction[a]
            t1 = (bmax[a] - origin[a]) / direction[a]
            t_enter = max(t_enter, min(t0, t1))
            t_exit = min(t_exit, max(t0, t1))
    return t_enter, t_exit


def center_depth(smoke, origin_m, cell_m, origin, direction, opacity, threshold) -> float:
    origin = np.asarray(origin, dtype=F)
    direction = np.asarray(direction, dtype=F)
    box_origin = np.asarray(origin_m, dtype=F)
    cell = F(cell_m)
    box_max = box_origin + np.asarray(smoke.shape, dtype=F) * cell
    s0, s1 = slab_range(origin, direction, box_origin, box_max)
    start = max(s0, F(0.0))
    found = F(-1.0)
    if s1 > start:
        length = F(s1 - start)
        steps = int(np.ceil(length / (F(0.5) * cell)))
        step_m = length / F(steps)
        transmittance = F(1.0)
        for s in range(steps):
            distance = start + (F(s) + F(0.5)) * step_m
            g = (origin + direction * distance - box_origin) / cell - F(0.5)
            density = max(sample(smoke, g), F(0.0))
            transmittance = transmittance * F(np.exp(np.float64(-F(opacity) * density * step_m)))
            if found < 0.0 and F(1.0) - transmittance >= F(threshold):
                found = distance
    return float(found)


def center_velocity(u, v, w) -> np.ndarray:
    return np.stack([F(0.5) * (u[:-1] + u[1:]), F(0.5) * (v[:, :-1] + v[:, 1:]), F(0.5) * (w[:, :, :-1] + w[:, :, 1:])],
                    axis=-1).astype(F)


def curl(centers: np.ndarray, cell_m: float) -> np.ndarray:
    c = centers.astype(F)
    n = c.shape[:3]
    grads = []
    for axis in range(3):
        idx = np.arange(n[axis])
        lo, hi = np.maximum(idx - 1, 0), np.minimum(idx + 1, n[axis] - 1)
        span = (hi - lo).astype(F)
        take_hi, take_lo = np.take(c, hi, axis=axis), np.take(c, lo, axis=axis)
        shape = [1, 1, 1, 1]
        shape[axis] = n[axis]
        span_b = span.reshape(shape)
        safe = np.where(span_b == 0, F(1.0), span_b * F(cell_m))
        grads.append(np.where(span_b == 0, F(0.0), (take_hi - take_lo) / safe))
    dx, dy, dz = grads
    return np.stack([dy[..., 2] - dz[..., 1], dz[..., 0] - dx[..., 2], dx[..., 1] - dy[..., 0]], axis=-1).astype(F)


def speed(vectors: np.ndarray) -> np.ndarray:
    v = vectors.astype(F)
    return np.sqrt((v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2])


def pixel_ray(view, px, py):
    right, up, toward = (np.asarray(getattr(view, k), dtype=F) for k in ("right", "up", "toward"))
    plane_x = F(view.left_m) + (F(px) + F(0.5)) * F(view.pixel_m)
    plane_y = F(view.top_m) - (F(py) + F(0.5)) * F(view.pixel_m)
    origin = (right * plane_x + up * plane_y) + toward * F(1.0e4)
    direction = -toward
    if view.perspective == 1:
        origin = np.asarray(view.eye, dtype=F)
        d = (right * plane_x + up * plane_y) - toward
        length = np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
        direction = d / length
    return origin, direction


def slice_overlay(view, origin_m, cell_m, axis, coordinate_m, values, low, high, ramp_table, image):
    out = image.copy()
    h, w = image.shape[:2]
    box_origin = np.asarray(origin_m, dtype=F)
    cell = F(cell_m)
    dims = values.shape
    for py in range(h):
        for px in range(w):
            origin, direction = pixel_ray(view, px, py)
            hit = False
            if abs(direction[axis]) > F(1.0e-9):
                distance = (F(coordinate_m) - origin[axis]) / direction[axis]
                if view.perspective == 0 or distance > F(0.0):
                    position = origin + direction * distance
                    hit = True
                    for other in range(3):
                        extent = F(dims[other]) * cell
                        if other != axis and (position[other] < box_origin[other]
                                              or position[other] > box_origin[other] + extent):
                            hit = False
            if hit:
                g = (position - box_origin) / cell - F(0.5)
                color = table_lookup(ramp_table, np.array([(sample(values, g) - F(low)) / (F(high) - F(low))]))[0]
                out[py, px, :3] = to_byte(color)
            else:
                out[py, px, :3] = to_byte(image[py, px, :3].astype(F) / F(255.0) * F(0.4))
    return out


def boundary_layers(smoke: np.ndarray) -> np.ndarray:
    side = max(smoke.shape)
    layers = np.zeros((6, side, side), dtype=np.float32)
    for face in range(6):
        axis = face // 2
        plane = np.take(smoke, (face % 2) * (smoke.shape[axis] - 1), axis=axis)
        layers[face, :plane.shape[0], :plane.shape[1]] = plane
    return layers
