"""The host option layers on the CPU: `DenoiserOptions.engine_spec` against the reference's
behavioural suite (av-denoise/src/host/tests/options.rs) and the VapourSynth parameter layer
against av-denoise-vs/tests/params.rs, restated on this package's API."""

import pytest

from conftest import avd


def raw(**kw):
    return dict(kw)


def opts(algorithm="nlmeans", **kw):
    return avd.vs_plane_options(raw(**kw), algorithm)


def error(algorithm="nlmeans", **kw):
    with pytest.raises(avd.InvalidOptions) as info:
        opts(algorithm, **kw)
    return str(info.value)


# ---- av-denoise/src/host/tests/options.rs ----

def gray_luma(**kw):
    return avd.DenoiserOptions(intent=avd.ChannelIntent.LUMA, chroma=avd.ChromaLayout.GRAY, **kw)


def test_default_algorithm_is_fast_nlmeans():
    o = gray_luma()
    assert o.algorithm.kind == "nlmeans" and o.algorithm.nlmeans == avd.NlmeansOptions()
    spec = o.engine_spec(32, 16)
    assert spec.luma.variant == avd.NlmeansVariant.FAST and spec.chroma is None


def test_geometry_carries_size_layout_and_depth():
    o = avd.DenoiserOptions(intent=avd.ChannelIntent.CHROMA, chroma=avd.ChromaLayout.YUV422, depth=avd.Depth.TEN)
    spec = o.engine_spec(32, 16)
    assert spec.luma is None and spec.chroma is not None
    g = spec.geometry
    assert (g.width, g.height, g.chroma) == (32, 16, avd.ChromaLayout.YUV422)
    assert g.input == g.output == avd.SampleFormat.u16(10)
    assert g.chroma_siting == avd.ChromaSiting.UNKNOWN
    spec.validate()


@pytest.mark.parametrize("intent,luma,chroma", [(avd.ChannelIntent.LUMA, True, False),
                                                (avd.ChannelIntent.CHROMA, False, True),
                                                (avd.ChannelIntent.LUMA_CHROMA, True, True)])
def test_each_intent_cleans_its_own_planes(intent, luma, chroma):
    for alg in (avd.Algorithm(), avd.Algorithm.nlmeans_hq(avd.NlmeansHqOptions()),
                avd.Algorithm.nl4d_options(avd.Nl4dOptions())):
        spec = avd.DenoiserOptions(intent=intent, chroma=avd.ChromaLayout.YUV420, algorithm=alg).engine_spec(64, 32)
        assert (spec.luma is not None, spec.chroma is not None) == (luma, chroma)


def test_mode_wins_over_the_algorithms_mode():
    fast = avd.NlmeansOptions(mode=avd.DenoisingMode.temporal(2))
    spec = gray_luma(algorithm=avd.Algorithm.nlmeans_fast(fast)).engine_spec(32, 16)
    assert spec.luma.options.mode == avd.DenoisingMode.spacial()
    hq = avd.NlmeansHqOptions(nlm=avd.NlmeansOptions(mode=avd.DenoisingMode.spacial()))
    spec = gray_luma(algorithm=avd.Algorithm.nlmeans_hq(hq), mode=avd.DenoisingMode.temporal(3)).engine_spec(32, 16)
    assert spec.luma.variant == avd.NlmeansVariant.HQ and spec.luma.options.mode == avd.DenoisingMode.temporal(3)


@pytest.mark.parametrize("mode,radius", [(avd.DenoisingMode.spacial(), 0), (avd.DenoisingMode.temporal(1), 1),
                                         (avd.DenoisingMode.temporal(4), 4)])
def test_mode_sets_the_nl4d_temporal_radius(mode, radius):
    spec = gray_luma(algorithm=avd.Algorithm.nl4d_options(avd.Nl4dOptions()), mode=mode).engine_spec(32, 16)
    assert spec.luma.temporal_radius == radius


def test_other_algorithm_options_pass_through():
    nl4d = avd.Nl4dOptions(sigma=0.02, refine=3, grain_data=True)
    spec = avd.DenoiserOptions(intent=avd.ChannelIntent.LUMA_CHROMA, chroma=avd.ChromaLayout.YUV420,
                               algorithm=avd.Algorithm.nl4d_options(nl4d),
                               mode=avd.DenoisingMode.temporal(2)).engine_spec(64, 32)
    for plane in (spec.luma, spec.chroma):
        assert plane.sigma == 0.02 and plane.refine == 3 and plane.grain_data


def test_per_plane_overrides():
    base = avd.NlmeansOptions(tuning=avd.NlmTuning(strength=1.0, search_radius=3))
    o = avd.DenoiserOptions(intent=avd.ChannelIntent.LUMA_CHROMA, chroma=avd.ChromaLayout.YUV420,
                            algorithm=avd.Algorithm.nlmeans_hq(avd.NlmeansHqOptions(nlm=base)),
                            luma_strength=0.6, chroma_sigma_scale=0.8)
    spec = o.engine_spec(64, 32)
    assert spec.luma.options.tuning.strength == 0.6 and spec.chroma.options.tuning.strength == 1.0
    assert spec.luma.options.tuning.search_radius == spec.chroma.options.tuning.search_radius == 3
    assert spec.luma.hq.sigma_scale == 1.0 and spec.chroma.hq.sigma_scale == 0.8
    n = avd.DenoiserOptions(intent=avd.ChannelIntent.LUMA_CHROMA, chroma=avd.ChromaLayout.YUV420,
                            algorithm=avd.Algorithm.nl4d_options(avd.Nl4dOptions(lambda_ht=3.0)),
                            chroma_lambda_ht=2.0, luma_lambda_ht_scale=1.2, luma_sigma_scale=1.3,
                            mode=avd.DenoisingMode.temporal(2)).engine_spec(64, 32)
    assert n.luma.lambda_ht == 3.0 and n.chroma.lambda_ht == 2.0
    assert n.luma.lambda_ht_scale == 1.2 and n.chroma.lambda_ht_scale == 1.0
    assert n.luma.sigma_scale == 1.3 and n.chroma.sigma_scale == 1.0
    unset = avd.DenoiserOptions(intent=avd.ChannelIntent.LUMA, chroma=avd.ChromaLayout.GRAY,
                                algorithm=avd.Algorithm.nl4d_options(avd.Nl4dOptions())).engine_spec(32, 16)
    assert unset.luma.lambda_ht is None


def test_depth_from_bits():
    assert [avd.Depth.from_bits(b) for b in (8, 10, 12, 16)] == [avd.Depth.EIGHT, avd.Depth.TEN, avd.Depth.TWELVE,
                                                                 avd.Depth.SIXTEEN]
    for bits in (0, 9, 14, 32):
        with pytest.raises(avd.InvalidOptions, match=f"unsupported integer bit depth {bits}"):
            avd.Depth.from_bits(bits)


# ---- av-denoise-vs/tests/params.rs: formats ----

@pytest.mark.parametrize("sw,sh,layout", [(1, 1, avd.ChromaLayout.YUV420), (1, 0, avd.ChromaLayout.YUV422),
                                          (0, 0, avd.ChromaLayout.YUV444)])
def test_layout_accepts_the_three_subsamplings(sw, sh, layout):
    assert avd.vs_layout_from_format("integer", 8, sw, sh, "yuv") == (layout, avd.Depth.EIGHT)
    assert avd.vs_layout_from_format("float", 32, sw, sh, "yuv") == (layout, avd.Depth.FLOAT)
    assert avd.vs_layout_from_format("integer", 16, sw, sh, "yuv")[1] == avd.Depth.SIXTEEN


def test_layout_rejections():
    def err(*a):
        with pytest.raises(avd.InvalidOptions) as info:
            avd.vs_layout_from_format(*a)
        return str(info.value)

    e = err("integer", 8, 0, 0, "RGB")
    assert "rgb" in e.lower() and "yuv" in e.lower()
    e = err("integer", 8, 0, 0, "gray")
    assert "gray" in e.lower() and "yuv" in e.lower()
    assert "gray" in err("float", 32, 0, 0, "gray").lower()
    assert "32-bit float" in err("float", 16, 1, 1, "yuv")
    assert "subsampling_w=2" in err("integer", 8, 2, 0, "yuv")
    assert "bit depth 9" in err("integer", 9, 1, 1, "yuv")


# ---- av-denoise-vs/tests/params.rs: parameters ----

def test_channel_mode():
    assert error(channel_mode="yuv") == "unknown channel_mode 'yuv', expected one of luma, chroma, lumachroma"
    assert opts(channel_mode="lumachroma").intent == avd.ChannelIntent.LUMA_CHROMA
    assert opts(channel_mode="Luma").intent == avd.ChannelIntent.LUMA


@pytest.mark.parametrize("name", ["strength", "patch_radius", "search_radius", "variant", "prefilter",
                                  "motion_compensation", "luma_strength", "chroma_strength"])
def test_nlm_only_params_are_rejected_for_nl4d(name):
    value = {"variant": "hq", "prefilter": "none", "motion_compensation": True}.get(name, 2)
    e = error("nl4d", **{name: value})
    assert name in e and "nl4d" in e


@pytest.mark.parametrize("name", ["luma_lambda_ht", "chroma_lambda_ht", "lambda_ht", "lambda_ht_scale",
                                  "luma_lambda_ht_scale", "chroma_lambda_ht_scale", "spatial_radius", "refine",
                                  "noise_map", "pooled_threshold"])
def test_nl4d_only_params_are_rejected_for_nlmeans(name):
    e = error(**{name: 1})
    assert name in e and "nlmeans" in e


def test_plane_params_for_a_plane_that_is_not_denoised():
    e = error(channel_mode="chroma", luma_strength=0.5)
    assert "luma_strength" in e and 'channel_mode="chroma"' in e
    assert "chroma_strength" in error(channel_mode="luma", chroma_strength=0.5)
    assert "chroma_lambda_ht_scale" in error("nl4d", channel_mode="luma", chroma_lambda_ht_scale=1.1)
    assert "luma_sigma_scale" in error("nl4d", channel_mode="chroma", luma_sigma_scale=1.1)
    assert opts(channel_mode="chroma", chroma_strength=0.3).chroma_strength == 0.3
    assert opts(channel_mode="luma", luma_strength=0.3).luma_strength == 0.3


def test_per_plane_overrides_reach_plane_options():
    o = opts(luma_strength=0.6, chroma_strength=0.3)
    assert (o.luma_strength, o.chroma_strength) == (0.6, 0.3)
    o = opts("nl4d", sigma_scale=1.1, luma_sigma_scale=1.3, chroma_sigma_scale=0.9, luma_lambda_ht_scale=1.2,
             chroma_lambda_ht_scale=0.8)
    assert (o.luma_sigma_scale, o.chroma_sigma_scale) == (1.3, 0.9)
    assert (o.luma_lambda_ht_scale, o.chroma_lambda_ht_scale) == (1.2, 0.8)
    assert o.algorithm.nl4d.sigma_scale == 1.1
    o = opts(variant="hq", luma_sigma_scale=1.3)
    assert (o.luma_sigma_scale, o.chroma_sigma_scale) == (1.3, None)


def test_sigma_and_sigma_scale():
    assert opts("nl4d", sigma=6.0).algorithm.nl4d.sigma == 6.0
    assert opts(variant="hq", sigma=6.0).algorithm.hq.sigma_override == 6.0
    assert opts(variant="hq", sigma_scale=1.5).algorithm.hq.sigma_scale == 1.5
    assert opts("nl4d", sigma_scale=1.5).algorithm.nl4d.sigma_scale == 1.5
    e = error(variant="fast", sigma=6.0)
    assert "sigma" in e and "fast" in e
    for name in ("sigma_scale", "luma_sigma_scale", "chroma_sigma_scale"):
        e = error(variant="fast", **{name: 1.2})
        assert name in e and "fast" in e


def test_variants():
    assert opts(variant="hq").algorithm.kind == "nlmeans_hq"
    assert opts(variant="fast").algorithm.kind == "nlmeans"
    assert opts(variant="HQ").algorithm.kind == "nlmeans_hq"
    assert opts().algorithm.kind == "nlmeans_hq"  # the base preset picks HQ
    e = error(variant="turbo")
    assert "turbo" in e and "fast" in e and "hq" in e


def test_temporal_radius():
    assert opts().mode == avd.DenoisingMode.temporal(2)
    assert opts(temporal_radius=0).mode == avd.DenoisingMode.spacial()
    assert opts(preset="veryfast", temporal_radius=3).mode == avd.DenoisingMode.temporal(3)
    assert "temporal_radius must not be negative, got -1" in error(temporal_radius=-1)


@pytest.mark.parametrize("name", ["veryfast", "fast", "base", "slow", "veryslow"])
def test_preset_resolves_the_same_dials_as_the_library(name):
    preset = avd.Preset[name.upper()]
    o = opts(preset=name)
    radius = avd.nlmeans_temporal_radius_for(preset)
    assert o.mode == (avd.DenoisingMode.spacial() if radius == 0 else avd.DenoisingMode.temporal(radius))
    hq = avd.nlmeans_variant_for(preset) == avd.NlmeansVariant.HQ
    assert (o.algorithm.kind == "nlmeans_hq") == hq
    assert o.algorithm.nlmeans.tuning.search_radius == avd.nlmeans_search_radius_for(preset)


def test_presets():
    assert opts(preset="BASE").mode == opts().mode
    e = error(preset="turbo")
    assert "turbo" in e
    assert opts(preset="veryfast", variant="hq").algorithm.kind == "nlmeans_hq"
    for name in ("veryfast", "fast", "veryslow"):
        assert "base and slow presets" in error("nl4d", preset=name)
    d = avd.Nl4dOptions()
    o = opts("nl4d", preset="base")
    assert o.mode == avd.DenoisingMode.temporal(d.temporal_radius)
    assert o.algorithm.nl4d.spatial_radius == d.spatial_radius


def test_motion_search_ceiling_follows_the_preset():
    assert opts("nl4d", preset="slow").algorithm.nl4d.motion.max_search_escalation == 8
    assert opts("nl4d", preset="base").algorithm.nl4d.motion.max_search_escalation == \
        avd.Nl4dOptions().motion.search_radius
    for preset, want in (("veryfast", 4), ("fast", 4), ("base", 4), ("slow", 8), ("veryslow", 8)):
        mc = opts(preset=preset, motion_compensation=True).algorithm.nlmeans.motion_compensation
        assert mc.search is not None and mc.search.max_search_escalation == want, preset


def test_motion_compensation_switch():
    assert opts().algorithm.nlmeans.motion_compensation.search is None
    assert opts(motion_compensation=False).algorithm.nlmeans.motion_compensation.search is None
    assert opts(motion_compensation=True).algorithm.nlmeans.motion_compensation.search is not None


def test_prefilter():
    assert opts(prefilter="none").algorithm.nlmeans.prefilter.kind == 0
    assert opts(prefilter="").algorithm.nlmeans.prefilter.kind == 0
    b = opts(prefilter="bilateral:3.0,0.02").algorithm.nlmeans.prefilter
    assert b.kind == 1 and abs(b.sigma_s - 3.0) < 1e-7 and abs(b.sigma_r - 0.02) < 1e-7
    assert opts(prefilter="nlm:0.8").algorithm.nlmeans.prefilter.strength_scale == 0.8
    with pytest.raises(ValueError):
        opts(prefilter="median")
    with pytest.raises(ValueError):
        opts(prefilter="external")


def test_nl4d_dials():
    base = opts("nl4d", preset="base").algorithm.nl4d
    assert opts("nl4d", spatial_radius=base.spatial_radius + 1).algorithm.nl4d.spatial_radius == \
        base.spatial_radius + 1
    assert opts("nl4d", refine=3).algorithm.nl4d.refine == 3
    assert base.noise_map and base.pooled_threshold
    assert not opts("nl4d", noise_map=False).algorithm.nl4d.noise_map
    assert not opts("nl4d", pooled_threshold=False).algorithm.nl4d.pooled_threshold
    assert abs(opts("nl4d", lambda_ht_scale=1.15).algorithm.nl4d.lambda_ht_scale - 1.15) < 1e-6
    assert opts("nl4d", lambda_ht=4.6).algorithm.nl4d.lambda_ht == 4.6
    assert "spatial_radius" in error("nl4d", spatial_radius=-2)


def test_tune_and_deterministic():
    o = opts()
    assert o.tuning == "auto" and not o.deterministic
    o = opts(tune=" Cached ", deterministic=True)
    assert o.tuning == "cached" and o.deterministic
    assert "sometimes" in error(tune="sometimes")


def test_plane_options_build_a_valid_engine_spec():
    """A resolved filter call becomes the engine spec the plugin would build: each plane takes its
    override and the spec validates."""
    o = opts(preset="fast", luma_strength=1.5, chroma_strength=0.8)
    layout, depth = avd.vs_layout_from_format("integer", 10, 1, 1, "yuv")
    spec = o.denoiser_options(layout, depth).engine_spec(64, 48)
    spec.validate()
    assert spec.luma.options.tuning.strength == 1.5 and spec.chroma.options.tuning.strength == 0.8
    assert spec.geometry.input == avd.SampleFormat.u16(10)
    n = opts("nl4d", luma_lambda_ht=3.0).denoiser_options(layout, depth).engine_spec(64, 48)
    n.validate()
    assert n.luma.lambda_ht == 3.0 and n.chroma.lambda_ht is None
