"""The VapourSynth filter's frame pump on the CPU: the reference's planner and packing tests
(av-denoise-vs/tests/stream.rs, tests/frames.rs) replayed on `av_denoise_b200.vs_filter`."""

import pytest

from conftest import avd
from av_denoise_b200 import vs_filter as vf

LOOKBACK, LEAD, LAST = 16, 2, 99


def geometry(edges, behind, ahead, last=LAST):
    return vf.StreamGeometry(avd.WindowSpan(behind, ahead, edges), LOOKBACK, LEAD, last)


def shifted():
    return geometry("shifted", 4, 4)


def repeat():
    return geometry("repeat", 2, 2)


class Harness:
    """stream.rs:37-144: drives a planner as the filter does, each output's index standing for it."""

    def __init__(self, g):
        self.planner = vf.StreamPlanner(g)
        self.outstanding = vf.Outstanding()
        self.buffer = vf.OutputBuffer()
        self.plans = []

    def register(self, frames):
        for n in frames:
            self.outstanding.register(n)

    def request(self, n):
        plan = self.planner.plan(n, self.buffer.contains(n), self.outstanding)
        if isinstance(plan, vf.Advance):
            self.run_steps(n, plan.steps)
        elif isinstance(plan, vf.Reseed):
            self.reseed(n, plan.start)
            self.run_steps(n, plan.steps)
        while not self.buffer.contains(n):
            index = self.planner.received()
            assert index is not None, "output n should be in flight"
            self.buffer.insert(index, index)
        assert self.buffer.take(n) == n
        self.buffer.evict_to(self.planner.geometry.buffer_capacity())
        self.outstanding.finish(n)
        self.plans.append(plan)
        return plan

    def reseed(self, n, start):
        g = self.planner.geometry
        rng = g.request_range(n)
        assert max(start - g.span.behind, 0) in rng
        assert min(start + g.span.ahead, g.last_frame) in rng
        self.buffer.insert(start, start)
        if g.reseed_ends_stream(start):
            for index in range(start + 1, g.last_frame + 1):
                self.buffer.insert(index, index)
        self.planner.reseeded(start)

    def run_steps(self, n, steps):
        g = self.planner.geometry
        rng = g.request_range(n)
        for step in steps:
            s = g.step(step)
            if isinstance(s, vf.Push):
                assert s.source in rng, f"pushed source {s.source} outside {rng}"
                self.planner.pushed()
            else:
                for index in self.planner.flushed():
                    self.buffer.insert(index, index)

    def reseeds(self):
        return sum(isinstance(p, vf.Reseed) for p in self.plans)


def render_in_order(h, frames):
    for n in frames:
        h.register([n])
        h.request(n)


def test_lookback_is_twice_the_thread_count_with_a_floor():
    assert vf.lookback_for(4) == vf.MIN_LOOKBACK and vf.lookback_for(32) == 64


def test_request_ranges_clamp_at_both_clip_ends():
    g = shifted()
    assert g.request_range(0) == range(0, 7)
    assert g.request_range(50) == range(30, 57)
    assert g.request_range(99) == range(79, 100)


def test_steps_flush_or_clamp_past_the_clip():
    assert shifted().step(95) == vf.Push(99) and shifted().step(96) == vf.Flush()
    assert repeat().step(97) == vf.Push(99) and repeat().step(99) == vf.Push(99)


def test_a_request_near_the_clip_start_reseeds_at_frame_zero():
    h = Harness(shifted())
    h.register([7])
    assert h.request(7) == vf.Reseed(0, range(1, 10))


@pytest.mark.parametrize("g", [shifted(), repeat(), geometry("shifted", 12, 12), geometry("repeat", 10, 10)])
def test_an_in_order_render_reseeds_once(g):
    h = Harness(g)
    render_in_order(h, range(LAST + 1))
    assert h.reseeds() == 1


def test_a_shuffled_burst_within_the_lookback_reseeds_once():
    h = Harness(shifted())
    h.register(range(16))
    for n in [9, 0, 13, 4, 5, 6, 1, 12, 2, 11, 3, 10, 7, 8, 15, 14]:
        h.request(n)
    assert h.reseeds() == 1


def test_a_burst_after_a_seek_reseeds_once_at_its_lowest_frame():
    h = Harness(shifted())
    h.register(range(50, 58))
    assert h.request(55) == vf.Reseed(50, range(51, 58))
    for n in [52, 50, 57, 51, 53, 56, 54]:
        h.request(n)
    assert h.reseeds() == 1


def test_a_single_scrub_and_a_request_behind_the_stream_reseed_at_the_frame():
    h = Harness(shifted())
    h.register([70])
    assert h.request(70) == vf.Reseed(70, range(71, 73))
    h = Harness(shifted())
    render_in_order(h, range(51))
    h.register([30])
    assert h.request(30) == vf.Reseed(30, range(31, 33))


def test_the_stream_catches_up_to_the_edge_of_the_request_range():
    h = Harness(shifted())
    render_in_order(h, range(11))
    assert h.planner.plan(37, False, h.outstanding) == vf.Advance(range(13, 40))
    assert h.planner.plan(38, False, h.outstanding) == vf.Reseed(38, range(39, 41))


def test_the_shifted_clip_end_flushes_and_serves_the_tail_from_the_buffer():
    h = Harness(shifted())
    render_in_order(h, range(95))
    assert h.plans[-1] == vf.Advance(range(96, 97))
    for n in range(95, LAST + 1):
        assert h.request(n) == vf.Serve()
    assert h.reseeds() == 1


def test_short_clips_flush_or_reseed_with_no_steps():
    h = Harness(geometry("shifted", 4, 4, 5))
    h.register(range(6))
    assert h.request(0) == vf.Reseed(0, range(1, 3))
    assert all(h.request(n) == vf.Serve() for n in range(1, 6))
    h = Harness(geometry("shifted", 4, 4, 2))
    h.register(range(3))
    assert h.request(0) == vf.Reseed(0, range(1, 1))
    assert all(h.request(n) == vf.Serve() for n in range(1, 3))


def test_a_killed_stream_reseeds_on_the_next_request():
    h = Harness(shifted())
    render_in_order(h, range(21))
    h.planner.kill()
    h.register([21])
    assert h.request(21) == vf.Reseed(21, range(22, 24))


@pytest.mark.parametrize("edges", ["shifted", "repeat"])
def test_every_plan_stays_inside_its_request_range(edges):
    h = Harness(geometry(edges, 4, 4))
    for first in range(0, LAST + 1, 8):
        last = min(first + 7, LAST)
        h.register(range(first, last + 1))
        for n in range(last, first - 1, -1):
            h.request(n)


def test_a_burst_wider_than_the_lookback_still_serves_every_frame():
    h = Harness(shifted())
    h.register(range(40))
    for n in range(39, -1, -1):
        h.request(n)
    assert h.reseeds() > 1


def test_outstanding_and_buffer_bookkeeping():
    o = vf.Outstanding()
    o.register(4)
    o.register(4)
    o.finish(4)
    assert o.lowest_in(0, 10) == 4
    o.finish(4)
    assert o.lowest_in(0, 10) is None
    o.finish(3)
    o.register(2)
    o.register(8)
    assert o.lowest_in(3, 10) == 8
    b = vf.OutputBuffer()
    for i in range(5):
        b.insert(i, i)
    b.evict_to(3)
    assert len(b) == 3 and not b.contains(1) and b.contains(2)
    b.insert(7, "seven")
    assert b.take(7) == "seven" and b.take(7) is None


def strided(width_bytes, height, stride):
    buf = bytearray([0xAA] * (stride * height))
    for y in range(height):
        for x in range(width_bytes):
            buf[y * stride + x] = (y * width_bytes + x) & 0xFF
    return bytes(buf)


def test_packing_drops_the_row_padding_and_round_trips():
    src = strided(5, 3, 8)
    packed = vf.pack_plane(src, 8, 5, 3)
    assert len(packed) == 15 and 0xAA not in packed
    assert list(packed) == list(range(15))
    dst = bytearray([0xAA] * 24)
    vf.unpack_plane_into(dst, 8, 5, 3, packed)
    assert bytes(dst) == src
    assert vf.pack_plane(strided(5, 3, 5), 5, 5, 3) == strided(5, 3, 5)
    two = vf.pack_plane(strided(8, 2, 12), 12, 8, 2)
    assert len(two) == 16 and 0xAA not in two


def test_window_indices_and_shifted_ranges():
    assert vf.window_indices(0, 2, 2, 11) == [0, 0, 0, 1, 2]
    assert vf.window_indices(1, 2, 2, 11) == [0, 0, 1, 2, 3]
    assert vf.window_indices(11, 2, 2, 11) == [9, 10, 11, 11, 11]
    assert vf.window_indices(10, 2, 2, 11) == [8, 9, 10, 11, 11]
    assert vf.window_indices(5, 2, 2, 11) == [3, 4, 5, 6, 7]
    assert vf.window_indices(1, 2, 2, 2) == [0, 0, 1, 2, 2]
    assert vf.window_indices(4, 0, 0, 11) == [4]
    assert vf.window_indices(5, 2, 4, 11) == [3, 4, 5, 6, 7, 8, 9]
    assert vf.window_indices(1, 2, 4, 11) == [0, 0, 1, 2, 3, 4, 5]
    assert vf.window_indices(9, 2, 4, 11) == [7, 8, 9, 10, 11, 11, 11]
    assert vf.shifted_window_range(0, 4, 4, 11) == range(0, 5)
    assert vf.shifted_window_range(2, 4, 4, 11) == range(0, 7)
    assert vf.shifted_window_range(11, 4, 4, 11) == range(7, 12)
    assert vf.shifted_window_range(9, 4, 4, 11) == range(5, 12)
    assert vf.shifted_window_range(6, 4, 4, 20) == range(2, 11)
    assert vf.shifted_window_range(1, 4, 4, 2) == range(0, 3)
