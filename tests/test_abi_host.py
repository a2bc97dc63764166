"""The C ABI library without a GPU: it loads, exports every symbol include/avd.h declares, and its
host-only entry points (defaults, presets, validation, window spans) match the reference."""

import ctypes as C
import re
from pathlib import Path

import pytest

from conftest import ROOT, avd

HEADER = ROOT / "include" / "avd.h"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(avd_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    # The Python mirror binds exactly the declared set.
    from av_denoise_b200 import _abi

    assert set(_abi.PROTOTYPES) == names


def test_abi_version(lib):
    assert lib.avd_abi_version() == 6


def test_status_messages(lib):
    assert lib.avd_status_message(4).decode() == "every ready frame must be emitted before the next push"
    assert lib.avd_status_message(7).decode().startswith("an earlier call failed")


def test_presets_match_reference():
    # nlmeans/options.rs:58-82, options.rs:170-175.
    P = avd.Preset
    assert [avd.nlmeans_variant_for(p) for p in P] == [0, 1, 1, 1, 1]
    assert [avd.nlmeans_temporal_radius_for(p) for p in P] == [0, 1, 2, 4, 8]
    assert [avd.nlmeans_search_radius_for(p) for p in P] == [2, 2, 2, 4, 4]
    assert [avd.search_escalation_for(p) for p in P] == [None, None, None, 8, 8]


def test_hq_default_strength_table():
    # nlmeans/params.rs:12-15.
    luma = [0.45, 0.45, 0.42, 0.42, 0.35, 0.35, 0.35, 0.30, 0.30]
    chroma = [1.00, 0.85, 0.70, 0.70, 0.70, 0.70, 0.70, 0.70, 0.70]
    for r in range(9):
        assert avd.hq_default_strength(1, r) == pytest.approx(luma[r])
        assert avd.hq_default_strength(2, r) == pytest.approx(chroma[r])
    assert avd.hq_default_strength(1, 20) == pytest.approx(0.30)


def test_defaults_match_reference(lib):
    from av_denoise_b200 import _abi

    n = _abi.AvdNl4dOptions()
    lib.avd_default_nl4d(C.byref(n))
    assert (n.refine, n.spatial_radius, n.temporal_radius) == (2, 9, 2)
    assert n.c_min == pytest.approx(0.05) and n.kaiser_beta == 2.0 and n.field_lambda == 1.0
    assert n.noise_map == 1 and n.pooled_threshold == 1 and n.grain_data == 0 and n.has_sigma == 0
    m = _abi.AvdMotionSearch()
    lib.avd_default_motion_search(C.byref(m))
    assert (m.blksize, m.overlap, m.search_radius, m.max_search_escalation, m.pyramid_levels) == (16, 8, 4, 4, 2)


def nlm(radius=None, **tuning):
    mode = avd.DenoisingMode.temporal(radius) if radius is not None else avd.DenoisingMode.spacial()
    return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=avd.NlmTuning(**tuning), mode=mode))


def geo(w=64, h=48, chroma=avd.ChromaLayout.YUV420, fmt=None, out=None):
    fmt = fmt or avd.SampleFormat.u8()
    return avd.Geometry(w, h, chroma, fmt, out or fmt)


def test_validate_accepts_plain_specs():
    avd.EngineSpec.nlmeans(nlm(2), None, geo()).validate()
    avd.EngineSpec.nlmeans(nlm(), nlm(), geo()).validate()
    avd.EngineSpec.nlmeans(nlm(1), nlm(1), geo(fmt=avd.SampleFormat.u16(10))).validate()


@pytest.mark.parametrize(
    "spec,err,text",
    [
        (lambda: avd.EngineSpec.nlmeans(None, None, geo()), avd.InvalidOptions, "clean luma, chroma or both"),
        (lambda: avd.EngineSpec.nlmeans(None, nlm(), geo(chroma=avd.ChromaLayout.GRAY)), avd.InvalidGeometry,
         "gray frame"),
        (lambda: avd.EngineSpec.nlmeans(nlm(), None, geo(fmt=avd.SampleFormat.u8(), out=avd.SampleFormat.u16(10))),
         avd.InvalidGeometry, "same input and output format"),
        (lambda: avd.EngineSpec.nlmeans(nlm(2), nlm(), geo()), avd.InvalidOptions, "chroma pass reads"),
        (lambda: avd.EngineSpec.nlmeans(nlm(search_radius=9), None, geo()), avd.InvalidOptions,
         "search_radius=9 exceeds"),
        (lambda: avd.EngineSpec.nlmeans(nlm(patch_radius=17), None, geo()), avd.InvalidOptions,
         "patch_radius=17 exceeds"),
        (lambda: avd.EngineSpec.nlmeans(nlm(9), None, geo()), avd.InvalidOptions, "temporal_radius=9 exceeds"),
        (lambda: avd.EngineSpec.nlmeans(nlm(strength=0.0), None, geo()), avd.InvalidOptions, "strength must be"),
        (lambda: avd.EngineSpec.nlmeans(nlm(self_weight=-1.0), None, geo()), avd.InvalidOptions, "self_weight"),
        (lambda: avd.EngineSpec.nlmeans(nlm(), None, geo(2, 2, avd.ChromaLayout.GRAY)), avd.InvalidGeometry,
         "below the supported minimum"),
        (lambda: avd.EngineSpec.nlmeans(nlm(), None, geo(fmt=avd.SampleFormat.u16(8))), avd.InvalidGeometry,
         "depth must be between 9 and 16"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(temporal_radius=0), None, geo()), avd.InvalidOptions,
         "temporal radius of at least 1"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(refine=5), None, geo()), avd.InvalidOptions, "refine=5"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(spatial_radius=17), None, geo()), avd.InvalidOptions,
         "spatial_radius=17"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(lambda_ht_scale=20.0), None, geo()), avd.InvalidOptions,
         "lambda_ht_scale"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(c_min=1.0), None, geo()), avd.InvalidOptions, "c_min"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(kaiser_beta=9.0), None, geo()), avd.InvalidOptions,
         "kaiser_beta"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(motion=avd.MotionSearch(blksize=16, overlap=14)), None, geo()),
         avd.InvalidOptions, "blocks cover a patch"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(motion=avd.MotionSearch(blksize=5)), None, geo()),
         avd.InvalidOptions, "must be even"),
        (lambda: avd.EngineSpec.nl4d(avd.Nl4dOptions(motion=avd.MotionSearch(max_search_escalation=2)), None,
                                     geo()), avd.InvalidOptions, "max_search_escalation"),
    ],
)
def test_validate_rejects_like_reference(spec, err, text):
    with pytest.raises(err, match=re.escape(text) if "=" in text else text):
        spec().validate()


def test_hq_sigma_scale_and_override_ranges():
    hq = avd.HqParams(sigma_scale=0.05)
    alg = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(hq=hq))
    with pytest.raises(avd.InvalidOptions, match="sigma_scale"):
        avd.EngineSpec.nlmeans(alg, None, geo()).validate()
    alg = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(hq=avd.HqParams.with_sigma(1.5)))
    with pytest.raises(avd.InvalidOptions, match="sigma_override"):
        avd.EngineSpec.nlmeans(alg, None, geo()).validate()


def test_window_spans():
    # engine/spec.rs:260-281: NLM holds d frames (plus the 8-frame look-ahead when HQ measures
    # noise); NL4D holds 2d (+ 8 when it measures noise) with shifted edges
    # (nl4d/tests/engine.rs:739-773).
    s = avd.EngineSpec.nlmeans(nlm(2), None, geo()).window_span()
    assert (s.behind, s.ahead, s.edges) == (2, 2, "repeat")
    hq = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=avd.NlmeansOptions(mode=avd.DenoisingMode.temporal(1))))
    s = avd.EngineSpec.nlmeans(hq, None, geo()).window_span()
    assert (s.behind, s.edges) == (9, "repeat")
    s = avd.EngineSpec.nl4d(avd.Nl4dOptions(temporal_radius=3), None, geo()).window_span()
    assert (s.behind, s.edges) == (14, "shifted")
    s = avd.EngineSpec.nl4d(avd.Nl4dOptions(temporal_radius=2), None, geo()).window_span()
    assert (s.behind, s.ahead) == (12, 12)
    s = avd.EngineSpec.nl4d(avd.Nl4dOptions(sigma=0.03), None, geo()).window_span()
    assert (s.behind, s.ahead) == (4, 4)


def test_create_validates_before_touching_the_gpu():
    # An invalid spec fails in build_engine with the reference's error, with no device needed.
    with pytest.raises(avd.InvalidOptions, match="search_radius=9"):
        avd.build_engine(avd.EngineSpec.nlmeans(nlm(search_radius=9), None, geo()))
