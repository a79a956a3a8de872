"""The reference's sheet-assembly property tests (tests/sheet/test_assemble.py in chadmv/plume) on the device
assembly: a square crop with an empty gutter in every frame, heat normalised to the hottest frame, frame
size and seat following the crop, an empty run refused, and packing order."""

import numpy as np
import pytest

from plume_b200.recipe.schema import NORMAL_LAYOUT, RenderSettings
from plume_b200.render.camera import make_camera, make_domain_view
from plume_b200.render.raw_frame import CHANNELS, HEAT, NORMAL_Z, THICKNESS

pytestmark = pytest.mark.gpu

VIEW = make_domain_view(make_camera(0.0, 0.0), (-1.0, 0.0, -1.0), (2.0, 2.0, 2.0), 0.0625, 2.0)  # 64 px
SOFT = RenderSettings(soften_px=0.75, crop_margin=0.04)


def disc(centre, radius, heat=0.0):
    frame = np.zeros((64, 64, CHANNELS), dtype=np.float32)
    frame[..., NORMAL_Z] = 1.0
    ys, xs = np.mgrid[0:64, 0:64] + 0.5
    inside = (xs - centre[0]) ** 2 + (ys - centre[1]) ** 2 < radius**2
    frame[inside, THICKNESS] = 0.8
    frame[inside, HEAT] = heat
    return frame


def rising():
    return [disc((32, 50 - 8 * i), 6 + 2 * i, heat=10.0 / (i + 1)) for i in range(4)]


def test_the_crop_is_square_and_every_frame_keeps_an_empty_gutter(cuda_device):
    from plume_b200.sheet.assemble import assemble

    result = assemble(rising(), VIEW, np.array([0.0, 0.2, 0.0]), 64, SOFT, NORMAL_LAYOUT)
    for frame in result.frames:
        assert frame.shape == (64, 64, 4)
        assert not frame[:2, :, :2].any() and not frame[-2:, :, :2].any()
        assert not frame[:, :2, :2].any() and not frame[:, -2:, :2].any()


def test_heat_is_normalised_to_the_hottest_frame(cuda_device):
    from plume_b200.sheet.assemble import assemble

    result = assemble(rising(), VIEW, np.array([0.0, 0.2, 0.0]), 64, SOFT, NORMAL_LAYOUT)
    assert max(int(frame[..., 0].max()) for frame in result.frames) == 255
    assert result.frames[0][..., 0].max() > result.frames[3][..., 0].max()


def test_the_frame_size_and_seat_follow_the_crop(cuda_device):
    from plume_b200.sheet.assemble import assemble

    result = assemble(rising(), VIEW, np.zeros(3), 64, RenderSettings(soften_px=0.0, crop_margin=0.0), NORMAL_LAYOUT)
    left, top, right, bottom = result.crop.box()
    assert right - left == pytest.approx(bottom - top)
    assert result.frame_m == pytest.approx(result.crop.side * VIEW.pixel_m)
    seat_x, seat_y = result.seat
    assert seat_x == pytest.approx(0.5, abs=0.02) and seat_y > 1.0  # centred on x = 0, the floor below


def test_a_run_with_nothing_visible_is_refused(cuda_device):
    from plume_b200.sheet.assemble import NothingVisibleError, assemble

    with pytest.raises(NothingVisibleError):
        assemble([np.zeros((64, 64, CHANNELS), dtype=np.float32)], VIEW, np.zeros(3), 64, SOFT, NORMAL_LAYOUT)


def test_packing_fills_rows_left_to_right_and_leaves_unused_slots_zero(cuda_device):
    import torch

    from plume_b200.sheet.assemble import pack

    frames = torch.stack([torch.full((4, 4, 4), index + 1, dtype=torch.uint8) for index in range(5)]).cuda()
    sheet = pack(frames, 3).cpu().numpy()
    assert sheet.shape == (8, 12, 4)
    assert sheet[0, 4, 0] == 2 and sheet[4, 0, 0] == 4 and not sheet[4:, 8:].any()


# ---- the shade layout (tests/sheet/test_shade_sheet.py) -----------------------------------------------------

def lit_ball(speckled_halo=False):
    """A dense ball lit from the left (shade 0.9 at its left edge to 0.3 at its right, stored times
    thickness); with a thin halo whose shade alternates 0.25 and 1 pixel by pixel when asked."""
    from plume_b200.render.raw_frame import SHADE

    frame = np.zeros((64, 64, CHANNELS), dtype=np.float32)
    ys, xs = np.mgrid[0:64, 0:64] + 0.5
    distance = np.hypot(xs - 32, ys - 32)
    ball = distance < 12
    frame[ball, THICKNESS] = 0.9
    frame[ball, SHADE] = 0.9 * (0.9 - 0.6 * (xs[ball] - 20) / 24)
    if speckled_halo:
        halo = (distance >= 12) & (distance < 18)
        checker = (np.floor(xs) + np.floor(ys)) % 2 == 0
        frame[halo, THICKNESS] = 0.02
        frame[halo, SHADE] = 0.02 * np.where(checker[halo], 0.25, 1.0)
    return frame


SEAT = np.array([0.0, 1.0, 0.0])


def shade_sheet(frames):
    from plume_b200.recipe.schema import SHADE_LAYOUT
    from plume_b200.sheet.assemble import assemble

    return assemble(frames, VIEW, SEAT, 64, RenderSettings(), SHADE_LAYOUT)


def test_every_alpha_byte_is_255(cuda_device):
    for frame in shade_sheet([lit_ball(speckled_halo=True), lit_ball()]).frames:
        assert np.all(frame[..., 3] == 255)


def test_empty_pixels_carry_their_neighbourhood_shade(cuda_device):
    frame = shade_sheet([lit_ball()]).frames[0]
    empty = frame[..., 1] == 0
    assert empty.any() and frame[empty, 2].min() > 0
    columns = np.arange(64)[None, :]
    assert frame[empty & (columns < 32), 2].mean() > frame[empty & (columns >= 32), 2].mean()


def test_a_speckled_thin_halo_is_smooth_and_no_darker_than_the_shaded_side(cuda_device):
    settings = RenderSettings()
    frame = shade_sheet([lit_ball(speckled_halo=True)]).frames[0]
    thickness = frame[..., 1].astype(np.float64) / 255.0
    shade = frame[..., 2].astype(np.float64)
    dense = thickness >= settings.shade_fade_thickness
    halo = (thickness > 0.0) & ~dense
    assert halo.any() and shade[halo].min() >= shade[dense].min() - 8
    neighbours = halo[:, 1:] & halo[:, :-1]
    assert np.abs(np.diff(shade, axis=1))[neighbours].max() <= 48


def test_the_brightest_well_covered_smoke_maps_to_255(cuda_device):
    settings = RenderSettings()
    result = shade_sheet([lit_ball()])
    frame = result.frames[0]
    dense = frame[..., 1] >= settings.shade_fade_thickness * 255
    assert frame[dense, 2].max() == 255 and result.shade_divisor == pytest.approx(0.9, abs=0.05)
