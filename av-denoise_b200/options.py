"""Host-side option layers above the engine spec, mirroring the reference's callers:

- `DenoiserOptions.engine_spec` follows av-denoise/src/host/options.rs:53-246: which planes a run
  cleans, its mode, its algorithm and the per-plane overrides become one `EngineSpec`.
- `vs_layout_from_format` and `vs_plane_options` follow av-denoise-vs/src/params.rs:44-518: a
  VapourSynth clip's format and a filter call's named arguments are checked and resolved the way the
  plugin resolves them, with the same error messages.

Both are pure host logic: they build specs and never touch the GPU."""

from __future__ import annotations

import enum
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence

from .api import (
    ChromaLayout,
    ChromaSiting,
    DenoisingMode,
    EngineSpec,
    Geometry,
    HqParams,
    InvalidOptions,
    MotionCompensationMode,
    MotionSearch,
    Nl4dOptions,
    NlmeansAlgorithm,
    NlmeansHqOptions,
    NlmeansOptions,
    NlmeansVariant,
    NlmTuning,
    PrefilterMode,
    Preset,
    SampleFormat,
    nlmeans_search_radius_for,
    nlmeans_temporal_radius_for,
    nlmeans_variant_for,
    parse_prefilter,
    search_escalation_for,
)


class ChannelIntent(enum.Enum):
    """av-denoise/src/host/options.rs:25-48: which planes a run cleans; the others pass through."""

    LUMA = "luma"
    CHROMA = "chroma"
    LUMA_CHROMA = "lumachroma"

    def cleans_luma(self) -> bool:
        return self in (ChannelIntent.LUMA, ChannelIntent.LUMA_CHROMA)

    def cleans_chroma(self) -> bool:
        return self in (ChannelIntent.CHROMA, ChannelIntent.LUMA_CHROMA)


class Depth(enum.Enum):
    """av-denoise/src/host/depth.rs:9-15: the wire bit depth of a run."""

    EIGHT = 8
    TEN = 10
    TWELVE = 12
    SIXTEEN = 16
    FLOAT = 32

    @staticmethod
    def from_bits(bits: int) -> "Depth":
        """depth.rs:22-35; the message of `UnsupportedDepthError`."""
        table = {8: Depth.EIGHT, 10: Depth.TEN, 12: Depth.TWELVE, 16: Depth.SIXTEEN}
        if bits not in table:
            raise InvalidOptions(f"unsupported integer bit depth {bits}, av-denoise supports 8, 10, 12, and 16-bit")
        return table[bits]

    def sample_format(self) -> SampleFormat:
        if self is Depth.FLOAT:
            return SampleFormat.f32()
        if self is Depth.EIGHT:
            return SampleFormat.u8()
        return SampleFormat.u16(self.value)


@dataclass
class Algorithm:
    """av-denoise/src/host/options.rs:248-261: `Nlmeans`, `NlmeansHq` or `Nl4d`, with the settings
    only that algorithm reads; the default is NLMeans with default options."""

    kind: str = "nlmeans"
    nlmeans: NlmeansOptions = field(default_factory=NlmeansOptions)
    hq: HqParams = field(default_factory=HqParams)
    nl4d: Nl4dOptions = field(default_factory=Nl4dOptions)

    @staticmethod
    def nlmeans_fast(options: NlmeansOptions) -> "Algorithm":
        return Algorithm("nlmeans", nlmeans=options)

    @staticmethod
    def nlmeans_hq(options: NlmeansHqOptions) -> "Algorithm":
        return Algorithm("nlmeans_hq", nlmeans=options.nlm, hq=options.hq)

    @staticmethod
    def nl4d_options(options: Nl4dOptions) -> "Algorithm":
        return Algorithm("nl4d", nl4d=options)


@dataclass
class DenoiserOptions:
    """av-denoise/src/host/options.rs:50-112 (`DenoiserOptions`)."""

    intent: ChannelIntent
    chroma: ChromaLayout
    mode: DenoisingMode = field(default_factory=DenoisingMode.spacial)
    algorithm: Algorithm = field(default_factory=Algorithm)
    luma_strength: Optional[float] = None
    chroma_strength: Optional[float] = None
    luma_lambda_ht: Optional[float] = None
    chroma_lambda_ht: Optional[float] = None
    luma_sigma_scale: Optional[float] = None
    chroma_sigma_scale: Optional[float] = None
    luma_lambda_ht_scale: Optional[float] = None
    chroma_lambda_ht_scale: Optional[float] = None
    depth: Depth = Depth.EIGHT
    chroma_siting: ChromaSiting = ChromaSiting.UNKNOWN
    tuning: str = "cached"
    deterministic: bool = False

    def temporal_radius(self) -> int:
        """options.rs:115-121."""
        return self.mode.radius or 0

    def engine_spec(self, width: int, height: int) -> EngineSpec:
        """options.rs:125-168: `mode` wins over whatever the algorithm holds; each plane group takes
        its own strength, `lambda_ht` and scale overrides."""
        fmt = self.depth.sample_format()
        geometry = Geometry(width, height, self.chroma, fmt, fmt, self.chroma_siting)
        luma, chroma = self.intent.cleans_luma(), self.intent.cleans_chroma()
        a = self.algorithm
        if a.kind == "nl4d":
            return EngineSpec.nl4d(self._plane_nl4d(True) if luma else None,
                                   self._plane_nl4d(False) if chroma else None, geometry)
        build = self._plane_hq if a.kind == "nlmeans_hq" else self._plane_fast
        return EngineSpec.nlmeans(build(True) if luma else None, build(False) if chroma else None, geometry)

    def _plane_nlm(self, luma: bool) -> NlmeansOptions:
        """options.rs:178-189 with `with_plane_strength` (options.rs:234-246)."""
        nlm = self.algorithm.nlmeans
        strength = self.luma_strength if luma else self.chroma_strength
        tuning = nlm.tuning if strength is None else replace(nlm.tuning, strength=strength)
        return replace(nlm, tuning=tuning, mode=self.mode)

    def _plane_fast(self, luma: bool) -> NlmeansAlgorithm:
        return NlmeansAlgorithm.fast(self._plane_nlm(luma))

    def _plane_hq(self, luma: bool) -> NlmeansAlgorithm:
        """options.rs:196-206: the plane's sigma_scale override wins over the algorithm's."""
        scale = self.luma_sigma_scale if luma else self.chroma_sigma_scale
        hq = self.algorithm.hq
        hq = replace(hq, sigma_scale=hq.sigma_scale if scale is None else scale)
        return NlmeansAlgorithm.hq_(NlmeansHqOptions(nlm=self._plane_nlm(luma), hq=hq))

    def _plane_nl4d(self, luma: bool) -> Nl4dOptions:
        """options.rs:208-226: the run's temporal radius; an unset `lambda_ht` stays unset, so the
        engine picks the plane's calibrated default."""
        nl4d = self.algorithm.nl4d
        lam = self.luma_lambda_ht if luma else self.chroma_lambda_ht
        scale = self.luma_sigma_scale if luma else self.chroma_sigma_scale
        lam_scale = self.luma_lambda_ht_scale if luma else self.chroma_lambda_ht_scale
        return replace(nl4d, temporal_radius=self.temporal_radius(),
                       lambda_ht=lam if lam is not None else nl4d.lambda_ht,
                       sigma_scale=nl4d.sigma_scale if scale is None else scale,
                       lambda_ht_scale=nl4d.lambda_ht_scale if lam_scale is None else lam_scale)


# ---- the VapourSynth plugin's parameter layer (av-denoise-vs/src/params.rs) ---------------------

def vs_layout_from_format(sample_type: str, bits_per_sample: int, subsampling_w: int, subsampling_h: int,
                          color_family: str) -> tuple[ChromaLayout, Depth]:
    """params.rs:44-97 (`layout_from_format`): YUV 4:2:0, 4:2:2 or 4:4:4 at 8, 10, 12 or 16-bit
    integer or 32-bit float. `sample_type` is "integer" or "float", `color_family` "yuv", "gray",
    "rgb" (or another VapourSynth family name)."""
    family = color_family.lower()
    if family == "gray":
        raise InvalidOptions(
            "GRAY clips are not supported, av-denoise-vs only accepts YUV420, YUV422, and YUV444 sources. Convert "
            "the input to YUV first, for example with `ffmpeg -pix_fmt yuv420p`")
    if family != "yuv":
        raise InvalidOptions(
            f"{color_family} clips are not supported, av-denoise's channel distance weights are calibrated for YUV. "
            "Convert the input to YUV first, for example with `ffmpeg -pix_fmt yuv420p`")
    if sample_type == "float":
        if bits_per_sample != 32:
            raise InvalidOptions(f"{bits_per_sample}-bit float clips are not supported, av-denoise-vs accepts 32-bit "
                                 "float or 8, 10, 12 and 16-bit integer YUV")
        depth = Depth.FLOAT
    else:
        depth = Depth.from_bits(bits_per_sample)
    layouts = {(0, 0): ChromaLayout.YUV444, (1, 0): ChromaLayout.YUV422, (1, 1): ChromaLayout.YUV420}
    if (subsampling_w, subsampling_h) not in layouts:
        raise InvalidOptions(f"unsupported chroma subsampling (subsampling_w={subsampling_w}, "
                             f"subsampling_h={subsampling_h}), av-denoise-vs accepts YUV420, YUV422, and YUV444")
    return layouts[(subsampling_w, subsampling_h)], depth


_PRESETS = {"veryfast": Preset.VERYFAST, "fast": Preset.FAST, "base": Preset.BASE, "slow": Preset.SLOW,
            "veryslow": Preset.VERYSLOW}
_NLM_ONLY = ("strength", "luma_strength", "chroma_strength", "patch_radius", "search_radius", "variant", "prefilter",
             "motion_compensation")
_NL4D_ONLY = ("luma_lambda_ht", "chroma_lambda_ht", "lambda_ht", "lambda_ht_scale", "luma_lambda_ht_scale",
              "chroma_lambda_ht_scale", "spatial_radius", "refine", "noise_map", "pooled_threshold", "wiener")
_KNOWN = set(_NLM_ONLY + _NL4D_ONLY + ("preset", "channel_mode", "device", "accelerators", "temporal_radius",
                                       "sigma", "sigma_scale", "tune", "deterministic", "luma_sigma_scale",
                                       "chroma_sigma_scale"))


@dataclass
class PlaneOptions:
    """av-denoise/src/planar/mod.rs:139-190 (`PlaneOptions`): a filter call's resolved settings."""

    intent: ChannelIntent
    mode: DenoisingMode
    algorithm: Algorithm
    device: Optional[str] = None
    accelerators: Optional[Sequence[str]] = None
    luma_strength: Optional[float] = None
    chroma_strength: Optional[float] = None
    luma_lambda_ht: Optional[float] = None
    chroma_lambda_ht: Optional[float] = None
    luma_sigma_scale: Optional[float] = None
    chroma_sigma_scale: Optional[float] = None
    luma_lambda_ht_scale: Optional[float] = None
    chroma_lambda_ht_scale: Optional[float] = None
    tuning: str = "auto"
    deterministic: bool = False

    def denoiser_options(self, chroma: ChromaLayout, depth: Depth) -> DenoiserOptions:
        return DenoiserOptions(intent=self.intent, chroma=chroma, mode=self.mode, algorithm=self.algorithm,
                               luma_strength=self.luma_strength, chroma_strength=self.chroma_strength,
                               luma_lambda_ht=self.luma_lambda_ht, chroma_lambda_ht=self.chroma_lambda_ht,
                               luma_sigma_scale=self.luma_sigma_scale, chroma_sigma_scale=self.chroma_sigma_scale,
                               luma_lambda_ht_scale=self.luma_lambda_ht_scale,
                               chroma_lambda_ht_scale=self.chroma_lambda_ht_scale, depth=depth,
                               tuning=self.tuning, deterministic=self.deterministic)


def _nonnegative(value: int, name: str) -> int:
    if value < 0:
        raise InvalidOptions(f"{name} must not be negative, got {value}")
    return int(value)


def vs_plane_options(raw: dict, algorithm: str) -> PlaneOptions:
    """params.rs:300-518 (`plane_options_from`) for `algorithm` "nlmeans" or "nl4d", over the filter
    call's named arguments `raw` (unset ones left out or None). The reference's check that a search
    radius above 4 needs a raised codegen stack belongs to its kernel compiler and has no
    counterpart here."""
    raw = {k: v for k, v in raw.items() if v is not None}
    unknown = sorted(set(raw) - _KNOWN)
    if unknown:
        raise InvalidOptions(f"unknown parameter {unknown[0]}")
    preset_name = raw.get("preset")
    if preset_name is None:
        preset = Preset.BASE
    elif preset_name.lower() in _PRESETS:
        preset = _PRESETS[preset_name.lower()]
    else:
        raise InvalidOptions(f"unknown preset '{preset_name}', expected one of veryfast, fast, base, slow, veryslow")
    if algorithm == "nl4d" and preset not in (Preset.BASE, Preset.SLOW):
        raise InvalidOptions("Nl4d only runs the base and slow presets, use temporal_radius and spatial_radius to "
                             "trade speed for quality")
    # params.rs:289-298 (`preset_motion_search`).
    defaults = MotionSearch()
    ceiling = search_escalation_for(preset) or defaults.search_radius
    motion = replace(defaults, max_search_escalation=max(ceiling, defaults.search_radius))
    if algorithm == "nlmeans":
        name = raw.get("variant")
        if name is None:
            variant = nlmeans_variant_for(preset)
        elif name.lower() in ("fast", "hq"):
            variant = NlmeansVariant.FAST if name.lower() == "fast" else NlmeansVariant.HQ
        else:
            raise InvalidOptions(f"unknown variant '{name}', expected one of fast, hq")
    else:
        variant = NlmeansVariant.HQ
    mode_name = raw.get("channel_mode")
    if mode_name is None:
        intent = ChannelIntent.LUMA_CHROMA
    else:
        try:
            intent = ChannelIntent(mode_name.lower())
        except ValueError:
            raise InvalidOptions(f"unknown channel_mode '{mode_name.lower()}', expected one of luma, chroma, "
                                 "lumachroma") from None
    # params.rs:164-262 (`reject_mismatched_params`).
    if algorithm == "nl4d":
        for name in _NLM_ONLY:
            if name in raw:
                raise InvalidOptions(f"{name} has no effect on nl4d, which has no NLM weighting pass to configure")
    else:
        for name in _NL4D_ONLY:
            if name in raw:
                raise InvalidOptions(f"{name} has no effect on nlmeans, which only nl4d reads")
        if variant == NlmeansVariant.FAST:
            if "sigma" in raw:
                raise InvalidOptions('sigma has no effect on nlmeans variant="fast", which has no noise measurement '
                                     'to pin. Set variant="hq" to use sigma')
            for name in ("sigma_scale", "luma_sigma_scale", "chroma_sigma_scale"):
                if name in raw:
                    raise InvalidOptions(f'{name} has no effect on nlmeans variant="fast", which has no noise '
                                         f'measurement to nudge. Set variant="hq" to use {name}')
    # params.rs:264-287 (`reject_unused_plane_params`).
    if intent != ChannelIntent.LUMA_CHROMA:
        unused, mode_label, plane = (("luma_strength", "luma_sigma_scale", "luma_lambda_ht_scale"), "chroma", "luma") \
            if intent == ChannelIntent.CHROMA else \
            (("chroma_strength", "chroma_sigma_scale", "chroma_lambda_ht_scale"), "luma", "chroma")
        for name in unused:
            if name in raw:
                raise InvalidOptions(f'{name} has no effect on channel_mode="{mode_label}", which does not denoise '
                                     f'{plane}')
    preset_radius = nlmeans_temporal_radius_for(preset) if algorithm == "nlmeans" else Nl4dOptions().temporal_radius
    if "temporal_radius" not in raw:
        mode = DenoisingMode.spacial() if preset_radius == 0 else DenoisingMode.temporal(preset_radius)
    else:
        r = _nonnegative(raw["temporal_radius"], "temporal_radius")
        mode = DenoisingMode.spacial() if r == 0 else DenoisingMode.temporal(r)
    if algorithm == "nlmeans":
        search_radius = _nonnegative(raw["search_radius"], "search_radius") if "search_radius" in raw \
            else nlmeans_search_radius_for(preset)
        tuning = NlmTuning(search_radius=search_radius,
                           patch_radius=_nonnegative(raw["patch_radius"], "patch_radius")
                           if "patch_radius" in raw else None,
                           strength=float(raw["strength"]) if "strength" in raw else None)
        mc = MotionCompensationMode(motion) if raw.get("motion_compensation") else MotionCompensationMode()
        prefilter = parse_prefilter(raw["prefilter"]) if "prefilter" in raw else PrefilterMode.none()
        nlm = NlmeansOptions(prefilter=prefilter, motion_compensation=mc, tuning=tuning, mode=mode)
        if variant == NlmeansVariant.FAST:
            alg = Algorithm.nlmeans_fast(nlm)
        else:
            hq = HqParams(sigma_override=float(raw["sigma"]) if "sigma" in raw else None,
                          sigma_scale=float(raw.get("sigma_scale", HqParams().sigma_scale)))
            alg = Algorithm.nlmeans_hq(NlmeansHqOptions(nlm=nlm, hq=hq))
    else:
        d = Nl4dOptions()
        alg = Algorithm.nl4d_options(Nl4dOptions(
            sigma=float(raw["sigma"]) if "sigma" in raw else None,
            sigma_scale=float(raw.get("sigma_scale", d.sigma_scale)),
            lambda_ht=float(raw["lambda_ht"]) if "lambda_ht" in raw else None,
            lambda_ht_scale=float(raw.get("lambda_ht_scale", d.lambda_ht_scale)),
            spatial_radius=_nonnegative(raw["spatial_radius"], "spatial_radius") if "spatial_radius" in raw
            else d.spatial_radius,
            refine=_nonnegative(raw["refine"], "refine") if "refine" in raw else d.refine,
            noise_map=bool(raw.get("noise_map", d.noise_map)),
            pooled_threshold=bool(raw.get("pooled_threshold", d.pooled_threshold)),
            wiener=bool(raw.get("wiener", d.wiener)),
            motion=motion))
    # tune/config.rs:22-38: trimmed and case-insensitive.
    text = raw.get("tune", "auto")
    tune = text.strip().lower()
    if tune not in ("auto", "cached", "off"):
        raise InvalidOptions(f"invalid tune: unknown tuning mode '{text}', expected auto, cached or off")

    def f(name):
        return float(raw[name]) if name in raw else None

    return PlaneOptions(intent=intent, mode=mode, algorithm=alg, device=raw.get("device"),
                        accelerators=raw.get("accelerators"), luma_strength=f("luma_strength"),
                        chroma_strength=f("chroma_strength"), luma_lambda_ht=f("luma_lambda_ht"),
                        chroma_lambda_ht=f("chroma_lambda_ht"), luma_sigma_scale=f("luma_sigma_scale"),
                        chroma_sigma_scale=f("chroma_sigma_scale"), luma_lambda_ht_scale=f("luma_lambda_ht_scale"),
                        chroma_lambda_ht_scale=f("chroma_lambda_ht_scale"), tuning=tune,
                        deterministic=bool(raw.get("deterministic", False)))
