"""Python mirror of av-denoise-core's public engine API, over the C ABI of libavd_b200.

Names, defaults and error behaviour follow the Rust crate (av-denoise-core/src/lib.rs:27-92):
`EngineSpec`, `Geometry`, `SampleFormat`, `ChromaLayout`, `DevicePlane`, `NlmeansAlgorithm`,
`NlmeansOptions`, `NlmeansHqOptions`, `HqParams`, `NlmTuning`, `DenoisingMode`, `Nl4dOptions`,
`MotionSearch`, `MotionEstimation`, `MotionCompensationMode`, `PrefilterMode`, `Preset`,
`build_engine`, and an `Engine` with push / push_context / emit_into / finish / reset.
Errors are raised as the `Error` variants of av-denoise-core/src/error.rs:3-19.
"""

from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Optional, Sequence

from . import _abi

# ---- errors (av-denoise-core/src/error.rs:3-19) ------------------------------------------------


class AvdError(Exception):
    status = -1


class InvalidOptions(AvdError):
    status = 1


class InvalidGeometry(AvdError):
    status = 2


class PlaneMismatch(AvdError):
    status = 3


class OutputsPending(AvdError):
    status = 4


class NothingToEmit(AvdError):
    status = 5


class ContextAfterPush(AvdError):
    status = 6


class NeedsReset(AvdError):
    status = 7


class GpuError(AvdError):
    status = 8


class QueueFull(AvdError):
    """av-denoise/src/host/mod.rs:40-44: MAX_PENDING frames wait to be collected; not poisoning."""

    status = 10


class Poisoned(AvdError):
    """av-denoise/src/host/mod.rs:45-49: an earlier call failed; reset the stream."""

    status = 11


_ERRORS = {c.status: c for c in (InvalidOptions, InvalidGeometry, PlaneMismatch, OutputsPending, NothingToEmit,
                                 ContextAfterPush, NeedsReset, GpuError, QueueFull, Poisoned)}


def _raise(status: int, message: str) -> None:
    if status == 0:
        return
    cls = _ERRORS.get(status, AvdError)
    raise cls(message or _abi.load().avd_status_message(status).decode())


# ---- geometry ----------------------------------------------------------------------------------


class ChromaLayout(enum.IntEnum):
    """engine/frame.rs:386-397."""

    GRAY = 0
    YUV420 = 1
    YUV422 = 2
    YUV444 = 3

    def plane_count(self) -> int:
        return 1 if self == ChromaLayout.GRAY else 3

    def chroma_dims(self, width: int, height: int) -> Optional[tuple[int, int]]:
        if self == ChromaLayout.GRAY:
            return None
        if self == ChromaLayout.YUV420:
            return (width + 1) // 2, (height + 1) // 2
        if self == ChromaLayout.YUV422:
            return (width + 1) // 2, height
        return width, height


class ChromaSiting(enum.IntEnum):
    LEFT = 0
    CENTER = 1
    TOP_LEFT = 2
    UNKNOWN = 3


@dataclass(frozen=True)
class SampleFormat:
    """engine/plane.rs:8-17: `U8`, `U16 { depth }` or `F32`."""

    kind: int
    depth: int = 0

    @staticmethod
    def u8() -> "SampleFormat":
        return SampleFormat(0, 8)

    @staticmethod
    def u16(depth: int) -> "SampleFormat":
        return SampleFormat(1, depth)

    @staticmethod
    def f32() -> "SampleFormat":
        return SampleFormat(2, 0)

    def max_value(self) -> float:
        return {0: 255.0, 1: float((1 << self.depth) - 1), 2: 1.0}[self.kind]

    def samples_per_word(self) -> int:
        return {0: 4, 1: 2, 2: 1}[self.kind]

    def plane_bytes(self, pixels: int) -> int:
        spw = self.samples_per_word()
        return (pixels + spw - 1) // spw * 4

    def _c(self) -> _abi.AvdSampleFormat:
        return _abi.AvdSampleFormat(self.kind, self.depth if self.kind == 1 else 0)


@dataclass
class Geometry:
    """engine/frame.rs:446-459."""

    width: int
    height: int
    chroma: ChromaLayout = ChromaLayout.YUV420
    input: SampleFormat = field(default_factory=SampleFormat.u8)
    output: SampleFormat = field(default_factory=SampleFormat.u8)
    chroma_siting: ChromaSiting = ChromaSiting.UNKNOWN

    def plane_dims(self, index: int) -> tuple[int, int]:
        if index == 0:
            return self.width, self.height
        dims = ChromaLayout(self.chroma).chroma_dims(self.width, self.height)
        return dims if dims else (self.width, self.height)

    def plane_count(self) -> int:
        return ChromaLayout(self.chroma).plane_count()

    def _c(self) -> _abi.AvdGeometry:
        return _abi.AvdGeometry(self.width, self.height, int(self.chroma), int(self.chroma_siting), self.input._c(),
                                self.output._c())


@dataclass
class DevicePlane:
    """engine/plane.rs:265-297: a borrowed, packed device plane (stride = width, whole words)."""

    ptr: int
    bytes: int
    width: int
    height: int

    @staticmethod
    def from_tensor(t, width: int, height: int) -> "DevicePlane":
        """Borrows a contiguous CUDA torch tensor as a plane."""
        if not t.is_cuda or not t.is_contiguous():
            raise PlaneMismatch("a device plane must be a contiguous CUDA tensor")
        return DevicePlane(t.data_ptr(), t.numel() * t.element_size(), width, height)

    def _c(self) -> _abi.AvdPlane:
        return _abi.AvdPlane(self.ptr, self.bytes, self.width, self.height)


# ---- options ------------------------------------------------------------------------------------


class Preset(enum.IntEnum):
    """options.rs:151-165."""

    VERYFAST = 0
    FAST = 1
    BASE = 2
    SLOW = 3
    VERYSLOW = 4


class NlmeansVariant(enum.IntEnum):
    FAST = 0
    HQ = 1


def nlmeans_variant_for(preset: Preset) -> NlmeansVariant:
    return NlmeansVariant(_abi.load().avd_nlmeans_variant_for(int(preset)))


def nlmeans_temporal_radius_for(preset: Preset) -> int:
    return int(_abi.load().avd_nlmeans_temporal_radius_for(int(preset)))


def nlmeans_search_radius_for(preset: Preset) -> int:
    return int(_abi.load().avd_nlmeans_search_radius_for(int(preset)))


def search_escalation_for(preset: Preset) -> Optional[int]:
    v = int(_abi.load().avd_search_escalation_for(int(preset)))
    return v or None


def hq_default_strength(channels: int, temporal_radius: int) -> float:
    """nlmeans/params.rs:27-33; channels 1 = luma, 2 = chroma."""
    return float(_abi.load().avd_hq_default_strength(channels, temporal_radius))


# nlmeans/prefilter/mod.rs:28-32: the pilot strength as a multiplier on the main pass strength.
DEFAULT_PILOT_STRENGTH_SCALE = 0.4


@dataclass
class PrefilterMode:
    """nlmeans/prefilter/mod.rs:15-26: kind 0 None, 1 Bilateral, 2 NlmSpatial."""

    kind: int = 0
    sigma_s: float = 0.0
    sigma_r: float = 0.0
    strength_scale: float = 0.0

    @staticmethod
    def none() -> "PrefilterMode":
        return PrefilterMode()

    @staticmethod
    def bilateral(sigma_s: float, sigma_r: float) -> "PrefilterMode":
        return PrefilterMode(1, sigma_s, sigma_r, 0.0)

    @staticmethod
    def nlm_spatial(strength_scale: float = DEFAULT_PILOT_STRENGTH_SCALE) -> "PrefilterMode":
        return PrefilterMode(2, 0.0, 0.0, strength_scale)

    def needs_reference_buf(self) -> bool:
        """nlmeans/prefilter/mod.rs:36-39: every prefilter keeps a reference ring."""
        return self.kind != 0

    def is_gpu_internal(self) -> bool:
        """nlmeans/prefilter/mod.rs:41-44: both prefilters build their reference on the GPU."""
        return self.kind in (1, 2)

    def _c(self) -> _abi.AvdPrefilter:
        return _abi.AvdPrefilter(self.kind, self.sigma_s, self.sigma_r, self.strength_scale)


def bilateral_radius(sigma_s: float) -> int:
    """nlmeans/prefilter/bilateral.rs:7-13: max(ceil(2 sigma_s), 1), evaluated in f32."""
    import numpy as np

    return max(int(np.ceil(np.float32(2.0) * np.float32(sigma_s))), 1)


def parse_prefilter(value: str) -> PrefilterMode:
    """nlmeans/prefilter/mod.rs:46-94 (`parse_prefilter`): "none" or "" -> None, "nlm" or
    "nlm:<strength_scale>" -> NlmSpatial, "bilateral:<sigma_s>,<sigma_r>" -> Bilateral. Raises
    ValueError on anything else, naming the form it expected."""
    if value in ("none", ""):
        return PrefilterMode.none()
    if value == "nlm":
        return PrefilterMode.nlm_spatial(DEFAULT_PILOT_STRENGTH_SCALE)
    if value.startswith("nlm:"):
        try:
            scale = float(value[4:].strip())
        except ValueError:
            raise ValueError("--prefilter nlm expects a number: nlm:<strength_scale>") from None
        return PrefilterMode.nlm_spatial(scale)
    if value.startswith("bilateral:"):
        parts = value[len("bilateral:"):].split(",")
        if len(parts) != 2:
            raise ValueError("--prefilter bilateral expects two values: bilateral:<sigma_s>,<sigma_r>")
        try:
            sigma_s, sigma_r = float(parts[0].strip()), float(parts[1].strip())
        except ValueError:
            raise ValueError("--prefilter bilateral expects two numbers: bilateral:<sigma_s>,<sigma_r>") from None
        return PrefilterMode.bilateral(sigma_s, sigma_r)
    raise ValueError(
        f"unknown prefilter '{value}', expected `none`, `nlm[:<strength_scale>]`, or `bilateral:<sigma_s>,<sigma_r>`")


class MotionEstimation(enum.IntEnum):
    AUTO = 0
    DIRECT = 1
    CHAINED = 2


@dataclass
class MotionSearch:
    """motion/search.rs:5-44."""

    blksize: int = 16
    overlap: int = 8
    search_radius: int = 4
    max_search_escalation: int = 4
    pyramid_levels: int = 2
    estimation: MotionEstimation = MotionEstimation.AUTO
    refine_radius: int = 2

    def _c(self) -> _abi.AvdMotionSearch:
        return _abi.AvdMotionSearch(self.blksize, self.overlap, self.search_radius, self.max_search_escalation,
                                    self.pyramid_levels, int(self.estimation), self.refine_radius)


@dataclass
class MotionCompensationMode:
    """motion/search.rs:58-89: `None` (search is None) or `Mvtools { .. }`."""

    search: Optional[MotionSearch] = None

    def _c(self) -> _abi.AvdMotionCompensation:
        s = self.search or MotionSearch()
        return _abi.AvdMotionCompensation(1 if self.search else 0, s._c())


@dataclass
class NlmTuning:
    """nlmeans/options.rs:94-101."""

    search_radius: Optional[int] = None
    patch_radius: Optional[int] = None
    strength: Optional[float] = None
    self_weight: Optional[float] = None

    def _c(self) -> _abi.AvdNlmTuning:
        def h(v):
            return (0, 0) if v is None else (1, v)

        sr, pr, st, sw = h(self.search_radius), h(self.patch_radius), h(self.strength), h(self.self_weight)
        return _abi.AvdNlmTuning(sr[0], sr[1], pr[0], pr[1], st[0], float(st[1]), sw[0], float(sw[1]))


@dataclass
class DenoisingMode:
    """nlmeans/options.rs:84-92: `Spacial` (radius None) or `Temporal { radius }`."""

    radius: Optional[int] = None

    @staticmethod
    def spacial() -> "DenoisingMode":
        return DenoisingMode(None)

    @staticmethod
    def temporal(radius: int) -> "DenoisingMode":
        return DenoisingMode(radius)

    def _c(self) -> _abi.AvdDenoisingMode:
        return _abi.AvdDenoisingMode(0 if self.radius is None else 1, self.radius or 0)


@dataclass
class HqParams:
    """nlmeans/params.rs:113-158."""

    auto_strength: bool = True
    noise_floor: bool = True
    sigma_override: Optional[float] = None
    temporal_confidence: bool = True
    thsad_scale: float = 1.0
    sigma_scale: float = 1.0

    @staticmethod
    def with_sigma(sigma: float) -> "HqParams":
        return HqParams(sigma_override=sigma)

    def _c(self) -> _abi.AvdHqParams:
        return _abi.AvdHqParams(int(self.auto_strength), int(self.noise_floor), int(self.sigma_override is not None),
                                float(self.sigma_override or 0.0), int(self.temporal_confidence), self.thsad_scale,
                                self.sigma_scale)


@dataclass
class NlmeansOptions:
    """nlmeans/options.rs:4-20."""

    prefilter: PrefilterMode = field(default_factory=PrefilterMode)
    motion_compensation: MotionCompensationMode = field(default_factory=MotionCompensationMode)
    tuning: NlmTuning = field(default_factory=NlmTuning)
    mode: DenoisingMode = field(default_factory=DenoisingMode)


@dataclass
class NlmeansHqOptions:
    """nlmeans/options.rs:22-29."""

    nlm: NlmeansOptions = field(default_factory=NlmeansOptions)
    hq: HqParams = field(default_factory=HqParams)


@dataclass
class NlmeansAlgorithm:
    """nlmeans/options.rs:41-46: `Fast(NlmeansOptions)` or `Hq(NlmeansHqOptions)`."""

    variant: NlmeansVariant
    options: NlmeansOptions
    hq: HqParams = field(default_factory=HqParams)

    @staticmethod
    def fast(options: NlmeansOptions) -> "NlmeansAlgorithm":
        return NlmeansAlgorithm(NlmeansVariant.FAST, options)

    @staticmethod
    def hq_(options: NlmeansHqOptions) -> "NlmeansAlgorithm":
        return NlmeansAlgorithm(NlmeansVariant.HQ, options.nlm, options.hq)

    def _c(self) -> _abi.AvdNlmeansAlgorithm:
        o = self.options
        return _abi.AvdNlmeansAlgorithm(int(self.variant), o.prefilter._c(), o.motion_compensation._c(),
                                        o.tuning._c(), o.mode._c(), self.hq._c())


@dataclass
class Nl4dOptions:
    """nl4d/options.rs:11-92."""

    motion: MotionSearch = field(default_factory=MotionSearch)
    sigma: Optional[float] = None
    sigma_scale: float = 1.0
    thsad_scale: float = 1.0
    refine: int = 2
    spatial_radius: int = 9
    lambda_ht: Optional[float] = None
    lambda_ht_scale: float = 1.0
    c_min: float = 0.05
    kaiser_beta: float = 2.0
    field_lambda: float = 1.0
    noise_map: bool = True
    pooled_threshold: bool = True
    grain_data: bool = False
    temporal_radius: int = 2
    # The empirical Wiener stage after the threshold: an extension, off by default (the reference's
    # filter stops at the threshold).
    wiener: bool = False

    def _c(self) -> _abi.AvdNl4dOptions:
        return _abi.AvdNl4dOptions(self.motion._c(), int(self.sigma is not None), float(self.sigma or 0.0),
                                   self.sigma_scale, self.thsad_scale, self.refine, self.spatial_radius,
                                   int(self.lambda_ht is not None), float(self.lambda_ht or 0.0),
                                   self.lambda_ht_scale, self.c_min, self.kaiser_beta, self.field_lambda,
                                   int(self.noise_map), int(self.pooled_threshold), int(self.grain_data),
                                   self.temporal_radius, int(self.wiener))


@dataclass
class EngineSpec:
    """engine/spec.rs:146-157: `Nlmeans { luma, chroma, geometry }` or `Nl4d { .. }`."""

    kind: int
    geometry: Geometry
    luma: object = None
    chroma: object = None

    @staticmethod
    def nlmeans(luma: Optional[NlmeansAlgorithm], chroma: Optional[NlmeansAlgorithm],
                geometry: Geometry) -> "EngineSpec":
        return EngineSpec(0, geometry, luma, chroma)

    @staticmethod
    def nl4d(luma: Optional[Nl4dOptions], chroma: Optional[Nl4dOptions], geometry: Geometry) -> "EngineSpec":
        return EngineSpec(1, geometry, luma, chroma)

    def _c(self) -> _abi.AvdEngineSpec:
        s = _abi.AvdEngineSpec()
        s.kind = self.kind
        s.has_luma = int(self.luma is not None)
        s.has_chroma = int(self.chroma is not None)
        lib = _abi.load()
        lib.avd_default_nlmeans(C.byref(s.nlm_luma))
        lib.avd_default_nlmeans(C.byref(s.nlm_chroma))
        lib.avd_default_nl4d(C.byref(s.nl4d_luma))
        lib.avd_default_nl4d(C.byref(s.nl4d_chroma))
        if self.kind == 0:
            if self.luma is not None:
                s.nlm_luma = self.luma._c()
            if self.chroma is not None:
                s.nlm_chroma = self.chroma._c()
        else:
            if self.luma is not None:
                s.nl4d_luma = self.luma._c()
            if self.chroma is not None:
                s.nl4d_chroma = self.chroma._c()
        s.geometry = self.geometry._c()
        return s

    def validate(self) -> None:
        """engine/spec.rs:291-345 plus the per-pass build checks; raises the matching error."""
        lib = _abi.load()
        buf = C.create_string_buffer(1024)
        st = lib.avd_spec_validate(C.byref(self._c()), buf, 1024)
        _raise(st, buf.value.decode())

    def window_span(self) -> "WindowSpan":
        out = _abi.AvdWindowSpan()
        _raise(_abi.load().avd_spec_window_span(C.byref(self._c()), C.byref(out)), "")
        return WindowSpan(out.behind, out.ahead, "shifted" if out.edges else "repeat")

    def max_held_frames(self) -> int:
        return self.window_span().behind


@dataclass
class WindowSpan:
    """engine/mod.rs:40-62."""

    behind: int
    ahead: int
    edges: str

    def frame_count(self) -> int:
        return self.behind + 1 + self.ahead


@dataclass
class EngineTiming:
    device_time: float
    frames: int
    exact_samples: int = 0  # samples the exact finish recomputed over the sampled frames
    core_time: float = 0.0  # the core launches' device time over the sampled frames (NL4D: search + filter)
    core_launches: int = 0


@dataclass
class PassTimings:
    luma: Optional[EngineTiming]
    chroma: Optional[EngineTiming]


# ---- engine -------------------------------------------------------------------------------------


def _planes(planes: Sequence[DevicePlane]):
    arr = (_abi.AvdPlane * max(1, len(planes)))()
    for i, p in enumerate(planes):
        arr[i] = p._c()
    return arr, len(planes)


class Engine:
    """engine/mod.rs:158-211 (`Engine`), through the C ABI."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._lib = _abi.load()

    def _check(self, status: int) -> None:
        if status:
            msg = self._lib.avd_engine_last_error(self._h)
            _raise(status, msg.decode() if msg else "")

    def set_stream(self, stream: int) -> None:
        """Queues every later call on CUDA stream `stream` (a `cudaStream_t` as an int)."""
        self._check(self._lib.avd_engine_set_stream(self._h, C.c_void_p(stream)))

    def push(self, planes: Sequence[DevicePlane]) -> int:
        arr, n = _planes(planes)
        ready = C.c_size_t(0)
        self._check(self._lib.avd_engine_push(self._h, arr, n, C.byref(ready)))
        return ready.value

    def push_context(self, planes: Sequence[DevicePlane]) -> None:
        arr, n = _planes(planes)
        self._check(self._lib.avd_engine_push_context(self._h, arr, n))

    def emit_into(self, planes: Sequence[DevicePlane]) -> None:
        arr, n = _planes(planes)
        self._check(self._lib.avd_engine_emit_into(self._h, arr, n))

    def finish(self) -> int:
        tail = C.c_size_t(0)
        self._check(self._lib.avd_engine_finish(self._h, C.byref(tail)))
        return tail.value

    def reset(self) -> None:
        self._check(self._lib.avd_engine_reset(self._h))

    def window_span(self) -> WindowSpan:
        out = _abi.AvdWindowSpan()
        self._check(self._lib.avd_engine_window_span(self._h, C.byref(out)))
        return WindowSpan(out.behind, out.ahead, "shifted" if out.edges else "repeat")

    def max_held_frames(self) -> int:
        out = C.c_size_t(0)
        self._check(self._lib.avd_engine_max_held_frames(self._h, C.byref(out)))
        return out.value

    def camera_models(self):
        """The camera-model ring after the queued work, (depth, 5) f32 (a, b, tx, ty, valid; stream
        frame f in row f % depth), or None when the engine fits no models (engine/spec.rs:403-415)."""
        import numpy as np

        depth = C.c_uint32(0)
        self._check(self._lib.avd_engine_models(self._h, None, 0, C.byref(depth)))
        if depth.value == 0:
            return None
        out = np.zeros(depth.value * 5, np.float32)
        self._check(self._lib.avd_engine_models(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size,
                                                C.byref(depth)))
        return out.reshape(depth.value, 5)

    def timing(self) -> PassTimings:
        out = _abi.AvdPassTimings()
        self._check(self._lib.avd_engine_timing(self._h, C.byref(out)))
        luma = (EngineTiming(out.luma.device_time, out.luma.frames, out.luma.exact_samples, out.luma.core_time,
                             out.luma.core_launches) if out.has_luma else None)
        chroma = (EngineTiming(out.chroma.device_time, out.chroma.frames, out.chroma.exact_samples,
                               out.chroma.core_time, out.chroma.core_launches)
                  if out.has_chroma else None)
        return PassTimings(luma, chroma)

    def sample_device_time(self, every: int) -> None:
        self._check(self._lib.avd_engine_sample_device_time(self._h, every))

    def fail_for_test(self) -> None:
        self._check(self._lib.avd_engine_fail_for_test(self._h))

    def close(self) -> None:
        if self._h:
            self._lib.avd_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


TUNING_MODES = {"auto": 0, "cached": 1, "off": 2}


def default_tuning_store() -> str:
    """The library's cache directory for tuning results: $XDG_CACHE_HOME/av-denoise-b200, else
    ~/.cache/av-denoise-b200 (created on first use)."""
    import os

    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    path = os.path.join(base, "av-denoise-b200")
    os.makedirs(path, exist_ok=True)
    return path


@dataclass
class TuningConfig:
    """tune/config.rs:8-75 (`TuningMode`, `TuningConfig`). `deterministic`: every NLMeans sample
    in the exact order of the reference's baseline, bit-identical to the CPU restatement on float
    outputs too (slower); integer outputs match it either way. `mode` ("auto", "cached" or "off")
    picks each launch site's variant per frame shape: auto times the variants once per shape and
    keeps the fastest. `store`: the directory results are kept in across processes (see
    `default_tuning_store`), or None for this process only."""

    deterministic: bool = False
    mode: str = "auto"
    store: Optional[str] = None

    def _c(self) -> _abi.AvdTuning:
        if self.mode not in TUNING_MODES:
            raise InvalidOptions(f"unknown tuning mode '{self.mode}', expected auto, cached or off")
        return _abi.AvdTuning(int(self.deterministic), TUNING_MODES[self.mode],
                              self.store.encode() if self.store else None)


def build_engine(spec: EngineSpec, tuning: Optional[TuningConfig] = None) -> Engine:
    """tune/setup.rs:79-91 (`build_engine`): validates, then builds on the current CUDA device."""
    lib = _abi.load()
    t = (tuning or TuningConfig())._c()
    h = C.c_void_p()
    st = lib.avd_engine_create(C.byref(spec._c()), C.byref(t), C.byref(h))
    if st:
        msg = lib.avd_last_error()
        _raise(st, msg.decode() if msg else "")
    return Engine(h)


# ---- host denoiser (av-denoise/src/host/mod.rs:111-420) ----------------------------------------

MAX_PENDING = 2  # av-denoise/src/host/mod.rs:27-28


@dataclass
class PlanarTiming:
    """av-denoise/src/host/timing.rs:20-36: host seconds blocked on readbacks and spent submitting,
    frames emitted, and each denoised plane group's device seconds (None when not sampled or not
    denoised)."""

    blocked: float
    submit: float
    frames: int
    luma: Optional[float]
    chroma: Optional[float]


class HostDenoiser:
    """A stateful denoiser over frames held as wire bytes, one buffer per plane (Y, then U and V).

    Mirrors `HostDenoiser` (av-denoise/src/host/mod.rs:111-420): `push` uploads a frame and starts
    any frame it completes; `recv` blocks for the oldest frame in flight (None when nothing is in
    flight); `flush` drains the frames in flight and the temporal tail into `sink`; `reset_stream`
    drops the stream and clears any poison. Raises `QueueFull` once MAX_PENDING frames wait, and
    `Poisoned` after a failure until `reset_stream`. Uploads and readbacks run natively in
    libavd_b200 (pinned staging, a copy stream, two output sets).
    """

    def __init__(self, spec: EngineSpec, tuning: Optional[TuningConfig] = None):
        self._lib = _abi.load()
        t = (tuning or TuningConfig())._c()
        h = C.c_void_p()
        st = self._lib.avd_host_create(C.byref(spec._c()), C.byref(t), C.byref(h))
        if st:
            msg = self._lib.avd_host_last_error(None)
            _raise(st, msg.decode() if msg else "")
        self._h = h
        self.spec = spec
        n = spec.geometry.plane_count()
        self.plane_lengths = [int(self._lib.avd_host_plane_bytes(h, i)) for i in range(n)]

    def _check(self, status: int) -> None:
        if status:
            msg = self._lib.avd_host_last_error(self._h)
            _raise(status, msg.decode() if msg else "")

    @staticmethod
    def _frame(planes: Sequence[bytes]):
        """Plane pointers without copies: bytes are passed in place, writable buffers by address;
        only a read-only buffer of another type is copied."""
        n = len(planes)
        ptrs = (C.c_void_p * max(1, n))()
        sizes = (_abi.u64 * max(1, n))()
        keep = []
        for i, p in enumerate(planes):
            if isinstance(p, bytes):
                ref = C.c_char_p(p)
                size = len(p)
            else:
                mv = memoryview(p).cast("B")
                size = len(mv)
                ref = (C.c_char * size).from_buffer_copy(mv) if mv.readonly else (C.c_char * size).from_buffer(mv)
            keep.append(ref)
            ptrs[i] = C.cast(ref, C.c_void_p)
            sizes[i] = size
        return ptrs, sizes, n, keep

    def push(self, planes: Sequence[bytes]) -> None:
        ptrs, sizes, n, _keep = self._frame(planes)
        self._check(self._lib.avd_host_push(self._h, ptrs, sizes, n))

    def push_priming(self, planes: Sequence[bytes]) -> None:
        ptrs, sizes, n, _keep = self._frame(planes)
        self._check(self._lib.avd_host_push_priming(self._h, ptrs, sizes, n))

    def recv(self) -> Optional[list[bytearray]]:
        bufs = [bytearray(n) for n in self.plane_lengths]
        return bufs if self.recv_into(bufs) else None

    def recv_into(self, out: Sequence) -> bool:
        """`recv` into caller-owned writable buffers (one per plane, each at least the plane's wire
        length); False when nothing was in flight."""
        views = [(C.c_char * n).from_buffer(memoryview(b).cast("B")) for b, n in zip(out, self.plane_lengths)]
        ptrs = (C.c_void_p * max(1, len(views)))(*[C.cast(v, C.c_void_p) for v in views])
        got = C.c_int(0)
        self._check(self._lib.avd_host_recv(self._h, ptrs, len(views), C.byref(got)))
        return bool(got.value)

    def flush(self, sink) -> None:
        lengths = self.plane_lengths
        failure: list[BaseException] = []

        def on_frame(_user, planes, n):
            if failure:
                return
            try:
                sink([C.string_at(planes[i], lengths[i]) for i in range(n)])
            except BaseException as e:  # re-raised after the native call returns
                failure.append(e)

        cb = _abi.AvdHostSink(on_frame)
        self._check(self._lib.avd_host_flush(self._h, cb, None))
        if failure:
            raise failure[0]

    def reset_stream(self) -> None:
        self._lib.avd_host_reset(self._h)

    def timing(self) -> PlanarTiming:
        t = _abi.AvdHostTiming()
        self._check(self._lib.avd_host_timing(self._h, C.byref(t)))

        def busy(has, v):
            return v if has and v >= 0 else None

        return PlanarTiming(t.blocked, t.submit, t.frames, busy(t.has_luma, t.luma_device_busy),
                            busy(t.has_chroma, t.chroma_device_busy))

    def sample_device_time(self, every: int) -> None:
        """Samples the device time of one frame in every `every`, or of none at 0."""
        self._lib.avd_host_sample_device_time(self._h, every)

    def poison_for_test(self) -> None:
        """Marks the stream failed, as mod.rs:392-395 does, to exercise `Poisoned` without a fault."""
        self._lib.avd_host_poison_for_test(self._h)

    def close(self) -> None:
        if self._h:
            self._lib.avd_host_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
