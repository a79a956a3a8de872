"""The frame cache's plan (tests/view/test_frame_cache.py in chadmv/plume): sizes, strides and when velocity
is dropped; host arithmetic only."""

from plume_b200.view.frame_cache import FrameCache, frame_bytes, frame_stride, keeps_velocity

CELLS = (8, 6, 4)


def test_the_stride_doubles_until_the_kept_frames_fit():
    one = frame_bytes(CELLS)
    assert one == 2 * 2 * 8 * 6 * 4
    assert frame_stride(64, CELLS, 64 * one) == 1
    assert frame_stride(64, CELLS, 64 * one - 1) == 2
    assert frame_stride(64, CELLS, 16 * one) == 4
    assert frame_stride(64, CELLS, 1) == 64  # one frame is always kept


def test_velocity_is_dropped_before_any_frame():
    with_velocity = frame_bytes(CELLS, velocity=True)
    assert with_velocity == 5 * 2 * 8 * 6 * 4
    assert keeps_velocity(8, CELLS, 8 * with_velocity) and not keeps_velocity(8, CELLS, 8 * with_velocity - 1)
    cache = FrameCache(CELLS, frames=8, budget_bytes=8 * with_velocity - 1, device="cuda:0")
    assert not cache.has_velocity and cache.stride == 1 and not cache.thinned
    assert "no velocity" in cache.thinning_note() and "every" not in cache.thinning_note()
    assert FrameCache(CELLS, frames=8, budget_bytes=8 * with_velocity, device="cuda:0").has_velocity


def test_nearest_kept_before_anything_lands_is_none():
    assert FrameCache(CELLS, frames=8, budget_bytes=1e9, device="cuda:0").nearest_kept(3) is None
