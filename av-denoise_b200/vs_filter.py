"""The VapourSynth filter's frame pump, above the host denoiser (av-denoise-vs/src/filter.rs,
stream.rs, frames.rs; av-denoise/src/planar/reseed.rs).

VapourSynth asks a filter for output frames in any order and from several threads. One denoiser
stream serves every request: a request for output n either finds n already buffered, catches the
live stream up (pushing source frames and receiving outputs until n lands), or rebuilds the stream
from a window of source frames around the lowest outstanding request near n (`reseed`). The
planner only holds indices; the filter runs each plan and reports every push, receive and flush so
the planner always matches the real stream.

VapourSynth itself is not a dependency: a source is any object with `num_frames`, the plane
geometry (`width`, `height`, `plane_dims(i)`, `bytes_per_sample`) and `get_frame(i)` returning
three `(bytes, stride)` planes, and `Denoise.get_frame` returns three packed planes written into
the caller's strided buffers by `unpack_plane_into`, as the plugin writes VapourSynth frames.
"""

from __future__ import annotations

import bisect
import threading
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

from . import api

MIN_LOOKBACK = 16  # stream.rs:7


# ---- frames.rs -------------------------------------------------------------------------------

def pack_plane(src: bytes, stride: int, width_bytes: int, height: int) -> bytes:
    """frames.rs:3-14: a plane with a row stride of `stride` bytes, packed tightly. `width_bytes` is
    width * bytes per sample, not a pixel count."""
    mv = memoryview(src)
    return b"".join(bytes(mv[y * stride:y * stride + width_bytes]) for y in range(height))


def unpack_plane_into(dst: bytearray, stride: int, width_bytes: int, height: int, src: bytes) -> None:
    """frames.rs:16-25: the packed plane `src` written back into `dst` (row stride `stride`);
    padding bytes are left untouched."""
    for y in range(height):
        dst[y * stride:y * stride + width_bytes] = src[y * width_bytes:(y + 1) * width_bytes]


def window_indices(output_index: int, behind: int, ahead: int, last_frame: int) -> list[int]:
    """frames.rs:27-35: the behind + 1 + ahead source indices around an output, clamped."""
    return [min(max(output_index + i - behind, 0), last_frame) for i in range(behind + ahead + 1)]


def shifted_window_range(output_index: int, behind: int, ahead: int, last_frame: int) -> range:
    """frames.rs:37-49: the source range around an output under shifted edges, cut at the clip's ends."""
    return range(max(output_index - behind, 0), min(output_index + ahead, last_frame) + 1)


# ---- stream.rs -------------------------------------------------------------------------------

def lookback_for(threads: int) -> int:
    """stream.rs:9-16: twice the worker threads, at least MIN_LOOKBACK."""
    return max(threads * 2, MIN_LOOKBACK)


@dataclass(frozen=True)
class Push:
    source: int


@dataclass(frozen=True)
class Flush:
    pass


@dataclass(frozen=True)
class Serve:
    pass


@dataclass(frozen=True)
class Advance:
    steps: range


@dataclass(frozen=True)
class Reseed:
    start: int
    steps: range


@dataclass(frozen=True)
class StreamGeometry:
    """stream.rs:39-102: the fixed shape of a filter's stream."""

    span: api.WindowSpan
    lookback: int
    lead: int
    last_frame: int

    def request_range(self, n: int) -> range:
        first = max(n - (self.span.behind + self.lookback), 0)
        last = min(n + self.span.ahead + self.lead, self.last_frame)
        return range(first, last + 1)

    def step(self, k: int):
        source = k + self.span.ahead
        if self.span.edges == "repeat":
            return Push(min(source, self.last_frame))
        return Push(source) if source <= self.last_frame else Flush()

    def reseed_ends_stream(self, start: int) -> bool:
        return self.span.edges == "shifted" and start + self.span.ahead >= self.last_frame

    def buffer_capacity(self) -> int:
        return self.lookback + self.span.frame_count() + self.lead

    def step_end(self, n: int) -> int:
        end = min(n + self.lead, self.last_frame) + 1
        if self.span.edges == "repeat":
            return end
        flush_step = max(self.last_frame + 1 - self.span.ahead, 0)
        return min(end, flush_step + 1)


class Outstanding:
    """stream.rs:251-281: output frames asked for and not yet given, counted per frame."""

    def __init__(self):
        self._counts: dict[int, int] = {}
        self._keys: list[int] = []

    def register(self, n: int) -> None:
        if n not in self._counts:
            bisect.insort(self._keys, n)
            self._counts[n] = 0
        self._counts[n] += 1

    def finish(self, n: int) -> None:
        if n not in self._counts:
            return
        self._counts[n] -= 1
        if self._counts[n] == 0:
            del self._counts[n]
            self._keys.pop(bisect.bisect_left(self._keys, n))

    def lowest_in(self, lo: int, hi: int) -> Optional[int]:
        i = bisect.bisect_left(self._keys, lo)
        return self._keys[i] if i < len(self._keys) and self._keys[i] <= hi else None


class OutputBuffer:
    """stream.rs:283-323: finished outputs waiting for their request."""

    def __init__(self):
        self._frames: dict[int, object] = {}

    def contains(self, index: int) -> bool:
        return index in self._frames

    def insert(self, index: int, frame) -> None:
        self._frames[index] = frame

    def take(self, index: int):
        return self._frames.pop(index, None)

    def evict_to(self, capacity: int) -> None:
        for index in sorted(self._frames)[:max(len(self._frames) - capacity, 0)]:
            del self._frames[index]

    def __len__(self) -> int:
        return len(self._frames)


class StreamPlanner:
    """stream.rs:110-249: decides how each request reaches its output, and tracks the stream."""

    def __init__(self, geometry: StreamGeometry):
        self.geometry = geometry
        self._live: Optional[tuple[int, int]] = None  # (next_step, next_output), or dead

    def plan(self, n: int, buffered: bool, outstanding: Outstanding):
        if buffered:
            return Serve()
        g = self.geometry
        end = g.step_end(n)
        if self._live is not None:
            next_step, next_output = self._live
            if next_output <= n and self._in_reach(next_step, n):
                return Advance(range(next_step, max(end, next_step)))
        floor = max(n - g.lookback, 0)
        lowest = outstanding.lowest_in(floor, n)
        start = 0 if floor == 0 else (lowest if lowest is not None else n)
        first_step = start + 1
        steps = range(first_step, first_step) if g.reseed_ends_stream(start) else range(first_step,
                                                                                       max(end, first_step))
        return Reseed(start, steps)

    def reseeded(self, start: int) -> None:
        self._live = None if self.geometry.reseed_ends_stream(start) else (start + 1, start + 1)

    def pushed(self) -> None:
        if self._live is not None:
            self._live = (self._live[0] + 1, self._live[1])

    def received(self) -> Optional[int]:
        if self._live is None:
            return None
        next_step, next_output = self._live
        if next_output >= next_step:
            return None
        self._live = (next_step, next_output + 1)
        return next_output

    def flushed(self) -> range:
        end = self.geometry.last_frame + 1
        first = self._live[1] if self._live is not None else end
        self._live = None
        return range(first, end)

    def kill(self) -> None:
        self._live = None

    def _in_reach(self, next_step: int, n: int) -> bool:
        step = self.geometry.step(next_step)
        return isinstance(step, Flush) or step.source >= self.geometry.request_range(n).start


# ---- planar/reseed.rs ------------------------------------------------------------------------

class PlanarDenoiser:
    """av-denoise/src/planar/mod.rs:277-610 and reseed.rs: a host denoiser over three wire planes,
    with the stream rebuilt from a window of source frames (`reseed`, `reseed_window`)."""

    def __init__(self, spec: api.EngineSpec, tuning: Optional[api.TuningConfig] = None):
        self.spec = spec
        self.host = api.HostDenoiser(spec, tuning)
        self.span = spec.window_span()

    def window_span(self) -> api.WindowSpan:
        return self.span

    def push(self, planes: Sequence[bytes]) -> None:
        self.host.push(planes)

    def recv(self):
        got = self.host.recv()
        return None if got is None else [bytes(p) for p in got]

    def flush(self, sink: Callable) -> None:
        self.host.flush(lambda planes: sink([bytes(p) for p in planes]))

    def reseed(self, window: Sequence[Sequence[bytes]]):
        """reseed.rs:47-99: the target of a mid-clip window of exactly span frames."""
        span = self.span
        if len(window) != span.frame_count():
            raise api.InvalidOptions(f"reseed needs a window of {span.frame_count()} frames, got {len(window)}")
        if span.edges == "shifted":
            outs = self.reseed_window(window, span.behind, False, False)
            return outs[-1]
        self.host.reset_stream()
        primed = span.behind + span.ahead
        for planes in window[:primed]:
            self.host.push_priming(planes)
        result = None
        for planes in window[primed:]:
            self.host.push(planes)
            got = self.recv()
            if got is not None:
                result = got
        if result is None:
            raise RuntimeError("a full window produced no frame")
        return result

    def reseed_window(self, frames: Sequence[Sequence[bytes]], target: int, at_clip_start: bool,
                      at_clip_end: bool) -> list:
        """reseed.rs:101-185: the target's output, and every later one when the window ends at the
        clip's end, from a window that stops at the clip's ends (shifted edges)."""
        span = self.span
        if span.edges != "shifted":
            raise api.InvalidOptions("reseed_window needs an algorithm with shifted edges, use reseed")
        if target >= len(frames):
            raise api.InvalidOptions(f"reseed target {target} is outside a window of {len(frames)}")
        ahead = len(frames) - 1 - target
        if target > span.behind or ahead > span.ahead:
            raise api.InvalidOptions("reseed window is longer than the span")
        want_ahead = ahead if at_clip_end else span.ahead
        want_behind = target if at_clip_start else span.behind
        if target != want_behind or len(frames) != want_behind + 1 + want_ahead:
            raise api.InvalidOptions("reseed window does not match the span for its edge flags")
        self.host.reset_stream()
        real = frames
        if not at_clip_start:
            for planes in frames[:span.behind]:
                self.host.push_priming(planes)
            real = frames[span.behind:]
        outputs = []
        for planes in real:
            self.host.push(planes)
            got = self.recv()
            if got is not None:
                outputs.append(got)
        if not at_clip_end:
            if not outputs:
                raise RuntimeError("a full window produced no frame")
            return [outputs[-1]]
        self.flush(outputs.append)
        from_end = len(frames) - target
        if len(outputs) < from_end:
            raise RuntimeError("a flushed window produced too few frames")
        return outputs[len(outputs) - from_end:]

    def close(self) -> None:
        self.host.close()


# ---- filter.rs -------------------------------------------------------------------------------

class Denoise:
    """filter.rs:59-519: `avd.NLMeans` / `avd.NL4D` over one denoiser stream shared by every request.

    `get_frame_initial(n)` registers the request and returns the source frames it needs;
    `get_frame(n)` renders output n (three packed planes). A failure kills the stream, so the next
    request rebuilds it. Two locks, as the plugin holds them: the outstanding requests (never held
    across GPU work) and the stream."""

    def __init__(self, source, spec: api.EngineSpec, threads: int = 8, tuning: Optional[api.TuningConfig] = None):
        self.source = source
        self.denoiser = PlanarDenoiser(spec, tuning)
        span = self.denoiser.window_span()
        self.geometry = StreamGeometry(span, lookback_for(threads), api.MAX_PENDING, source.num_frames - 1)
        self.planner = StreamPlanner(self.geometry)
        self.buffer = OutputBuffer()
        self.outstanding = Outstanding()
        self._outstanding_lock = threading.Lock()
        self._state_lock = threading.Lock()

    # -- the source frames (packed wire planes) --
    def _fetch(self, index: int):
        planes = self.source.get_frame(index)
        bps = self.source.bytes_per_sample
        out = []
        for i, (data, stride) in enumerate(planes):
            w, h = self.source.plane_dims(i)
            out.append(pack_plane(data, stride, w * bps, h))
        return out

    def get_frame_initial(self, n: int) -> range:
        with self._outstanding_lock:
            self.outstanding.register(n)
        return self.geometry.request_range(n)

    def get_frame(self, n: int):
        try:
            return self._render(n)
        finally:
            with self._outstanding_lock:
                self.outstanding.finish(n)

    def _render(self, n: int):
        with self._state_lock:
            try:
                return self._render_locked(n)
            except BaseException:
                self.planner.kill()
                raise

    def _render_locked(self, n: int):
        buffered = self.buffer.contains(n)
        with self._outstanding_lock:
            plan = self.planner.plan(n, buffered, self.outstanding)
        if isinstance(plan, Advance):
            self._run_steps(plan.steps)
        elif isinstance(plan, Reseed):
            self._reseed_at(plan.start)
            self._run_steps(plan.steps)
        self._receive_all()
        out = self.buffer.take(n)
        if out is None:
            raise RuntimeError(f"output frame {n} was never produced")
        self.buffer.evict_to(self.geometry.buffer_capacity())
        return out

    def _reseed_at(self, start: int) -> None:
        span, last = self.geometry.span, self.geometry.last_frame
        if span.edges == "repeat":
            window = [self._fetch(i) for i in window_indices(start, span.behind, span.ahead, last)]
            self.buffer.insert(start, self.denoiser.reseed(window))
            self.planner.reseeded(start)
            return
        rng = shifted_window_range(start, span.behind, span.ahead, last)
        window = [self._fetch(i) for i in rng]
        outs = self.denoiser.reseed_window(window, start - rng.start, rng.start == 0, rng.stop - 1 == last)
        for offset, planes in enumerate(outs):
            self.buffer.insert(start + offset, planes)
        self.planner.reseeded(start)

    def _run_steps(self, steps: range) -> None:
        for step in steps:
            s = self.geometry.step(step)
            if isinstance(s, Push):
                self._push_with_drain(self._fetch(s.source))
            else:
                self._flush_into_buffer()

    def _push_with_drain(self, planes) -> None:
        try:
            self.denoiser.push(planes)
        except api.QueueFull:
            self._receive_one()
            self.denoiser.push(planes)
        self.planner.pushed()

    def _receive_one(self) -> None:
        index = self.planner.received()
        if index is None:
            raise RuntimeError("no output is in flight to receive")
        self._receive_output(index)

    def _receive_all(self) -> None:
        while (index := self.planner.received()) is not None:
            self._receive_output(index)

    def _receive_output(self, index: int) -> None:
        got = self.denoiser.recv()
        if got is None:
            raise RuntimeError(f"the stream yielded nothing for output {index}")
        self.buffer.insert(index, got)

    def _flush_into_buffer(self) -> None:
        outputs = []
        self.denoiser.flush(outputs.append)
        indices = self.planner.flushed()
        if len(outputs) != len(indices):
            raise RuntimeError(f"the clip's final flush produced {len(outputs)} frames, expected {len(indices)}")
        for index, planes in zip(indices, outputs):
            self.buffer.insert(index, planes)

    def close(self) -> None:
        self.denoiser.close()
