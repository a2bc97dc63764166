"""ctypes mirror of include/avd.h.

The structures here are byte-for-byte the C structs; `load()` binds every exported function with
its prototype. Nothing here falls back to Python arithmetic: without the built library, `load()`
raises.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libavd_b200.so"

u32 = C.c_uint32
u64 = C.c_uint64
f32 = C.c_float


class AvdSampleFormat(C.Structure):
    _fields_ = [("kind", u32), ("depth", u32)]


class AvdGeometry(C.Structure):
    _fields_ = [
        ("width", u32),
        ("height", u32),
        ("chroma", u32),
        ("chroma_siting", u32),
        ("input", AvdSampleFormat),
        ("output", AvdSampleFormat),
    ]


class AvdPlane(C.Structure):
    _fields_ = [("ptr", u64), ("bytes", u64), ("width", u32), ("height", u32)]


class AvdPrefilter(C.Structure):
    _fields_ = [("kind", u32), ("sigma_s", f32), ("sigma_r", f32), ("strength_scale", f32)]


class AvdMotionSearch(C.Structure):
    _fields_ = [
        ("blksize", u32),
        ("overlap", u32),
        ("search_radius", u32),
        ("max_search_escalation", u32),
        ("pyramid_levels", u32),
        ("estimation", u32),
        ("refine_radius", u32),
    ]


class AvdMotionCompensation(C.Structure):
    _fields_ = [("active", u32), ("search", AvdMotionSearch)]


class AvdNlmTuning(C.Structure):
    _fields_ = [
        ("has_search_radius", u32),
        ("search_radius", u32),
        ("has_patch_radius", u32),
        ("patch_radius", u32),
        ("has_strength", u32),
        ("strength", f32),
        ("has_self_weight", u32),
        ("self_weight", f32),
    ]


class AvdDenoisingMode(C.Structure):
    _fields_ = [("temporal", u32), ("radius", u32)]


class AvdHqParams(C.Structure):
    _fields_ = [
        ("auto_strength", u32),
        ("noise_floor", u32),
        ("has_sigma_override", u32),
        ("sigma_override", f32),
        ("temporal_confidence", u32),
        ("thsad_scale", f32),
        ("sigma_scale", f32),
    ]


class AvdNlmeansAlgorithm(C.Structure):
    _fields_ = [
        ("variant", u32),
        ("prefilter", AvdPrefilter),
        ("motion_compensation", AvdMotionCompensation),
        ("tuning", AvdNlmTuning),
        ("mode", AvdDenoisingMode),
        ("hq", AvdHqParams),
    ]


class AvdNl4dOptions(C.Structure):
    _fields_ = [
        ("motion", AvdMotionSearch),
        ("has_sigma", u32),
        ("sigma", f32),
        ("sigma_scale", f32),
        ("thsad_scale", f32),
        ("refine", u32),
        ("spatial_radius", u32),
        ("has_lambda_ht", u32),
        ("lambda_ht", f32),
        ("lambda_ht_scale", f32),
        ("c_min", f32),
        ("kaiser_beta", f32),
        ("field_lambda", f32),
        ("noise_map", u32),
        ("pooled_threshold", u32),
        ("grain_data", u32),
        ("temporal_radius", u32),
        ("wiener", u32),
    ]


class AvdEngineSpec(C.Structure):
    _fields_ = [
        ("kind", u32),
        ("has_luma", u32),
        ("has_chroma", u32),
        ("nlm_luma", AvdNlmeansAlgorithm),
        ("nlm_chroma", AvdNlmeansAlgorithm),
        ("nl4d_luma", AvdNl4dOptions),
        ("nl4d_chroma", AvdNl4dOptions),
        ("geometry", AvdGeometry),
    ]


class AvdTuning(C.Structure):
    _fields_ = [("deterministic", u32), ("mode", u32), ("store", C.c_char_p)]


class AvdWindowSpan(C.Structure):
    _fields_ = [("behind", u64), ("ahead", u64), ("edges", u32), ("reserved", u32)]


class AvdEngineTiming(C.Structure):
    _fields_ = [("device_time", C.c_double), ("frames", u64), ("exact_samples", u64), ("core_time", C.c_double),
                ("core_launches", u64)]


class AvdPassTimings(C.Structure):
    _fields_ = [("has_luma", u32), ("has_chroma", u32), ("luma", AvdEngineTiming), ("chroma", AvdEngineTiming)]


class AvdCollabPass(C.Structure):
    _fields_ = [(n, u64) for n in ("ring", "mv_field", "confidence", "neighbour_slots", "noise", "noise_curve",
                                   "dct_profile", "kaiser", "accum", "wsum", "group_weight", "members")] + \
               [(n, u32) for n in ("width", "height", "channels", "centre_slot", "sigma_word", "weight_scale_word",
                                   "curve_valid_word", "radius", "refine", "spatial_radius", "k_max", "mv_stride",
                                   "conf_stride", "blk_step", "blksize", "blocks_x", "blocks_y", "pooled")] + \
               [(n, f32) for n in ("c_min", "lambda_ht", "accum_scale", "pool_ratio")] + [("wiener", u32)]


class AvdBatchIngest(C.Structure):
    _fields_ = [(n, u64) for n in ("plane0", "plane1", "frame")] + [(n, u32) for n in ("width", "height", "channels",
                                                                                       "bits")]


class AvdCollabAdjoint(C.Structure):
    _fields_ = [(n, u64) for n in ("grad_accum", "grad_wsum", "grad_ring", "grad_sigma_refs")]


class AvdMotionPass(C.Structure):
    _fields_ = [(n, u64) for n in ("pyramid", "neighbour_slots", "mv_field", "confidence", "noise")] + \
               [(n, u32) for n in ("width", "height", "frame_count", "centre_slot", "neighbours", "blksize", "overlap",
                                   "search_radius", "levels", "mv_stride", "conf_stride", "sad_floor_word")] + \
               [("thsad", f32), ("seeded", u32), ("keep_seeds", u64), ("escalation", u64), ("ceiling", u32),
                ("esc_reads_floor", u32), ("predictions", u64), ("sad", u64), ("coarse_radius", u32),
                ("coarse_block_factor", u32)]


class AvdTruemotionPass(C.Structure):
    _fields_ = [(n, u64) for n in ("pyramid", "neighbour_slots", "mv_in", "seeds", "mv_out", "confidence",
                                   "noise")] + \
               [(n, u32) for n in ("width", "height", "frame_count", "centre_slot", "neighbours", "blksize", "overlap",
                                   "mv_stride", "conf_stride", "sad_field", "reads_floor")] + \
               [("field_lambda", f32), ("thsad", f32), ("predictions", u64), ("sad", u64)]


class AvdModelFit(C.Structure):
    _fields_ = [("field", u64), ("sad", u64)] + \
               [(n, u32) for n in ("has_contrast", "means_offset", "older_to_newer", "width", "height", "blksize",
                                   "overlap")] + \
               [("prior", C.c_int32), ("models", u64), ("slot", u32), ("scratch", u64)]


class AvdNlmBackward(C.Structure):
    _fields_ = [(n, u64) for n in ("window", "grad_out", "grad_window", "grad_strength", "scratch")] + \
               [(n, u32) for n in ("width", "height", "channels", "temporal_radius", "search_radius",
                                   "patch_radius")] + \
               [(n, f32) for n in ("strength", "self_weight", "pair_offset", "spatial_offset")]


class AvdBatchJob(C.Structure):
    _fields_ = [("frames", u64), ("out", u64)] + \
               [(n, u32) for n in ("n_frames", "centre", "temporal_radius", "width", "height")] + \
               [(n, f32) for n in ("strength", "pair_offset", "spatial_offset")]


class AvdHostTiming(C.Structure):
    _fields_ = [("blocked", C.c_double), ("submit", C.c_double), ("frames", u64), ("has_luma", u32),
                ("has_chroma", u32), ("luma_device_busy", C.c_double), ("chroma_device_busy", C.c_double)]


_P = C.POINTER
_E = C.c_void_p  # AvdEngine*
_H = C.c_void_p  # AvdHost*
# void (*AvdHostSink)(void* user, const void* const* planes, size_t n)
AvdHostSink = C.CFUNCTYPE(None, C.c_void_p, _P(C.c_void_p), C.c_size_t)

# name -> (restype, argtypes); the exact set of entry points include/avd.h declares.
PROTOTYPES: dict[str, tuple] = {
    "avd_abi_version": (u32, []),
    "avd_status_message": (C.c_char_p, [C.c_int]),
    "avd_default_nlmeans": (None, [_P(AvdNlmeansAlgorithm)]),
    "avd_default_nl4d": (None, [_P(AvdNl4dOptions)]),
    "avd_default_motion_search": (None, [_P(AvdMotionSearch)]),
    "avd_nlmeans_variant_for": (u32, [u32]),
    "avd_nlmeans_temporal_radius_for": (u32, [u32]),
    "avd_nlmeans_search_radius_for": (u32, [u32]),
    "avd_search_escalation_for": (u32, [u32]),
    "avd_hq_default_strength": (f32, [u32, u32]),
    "avd_spec_validate": (C.c_int, [_P(AvdEngineSpec), C.c_char_p, C.c_size_t]),
    "avd_spec_window_span": (C.c_int, [_P(AvdEngineSpec), _P(AvdWindowSpan)]),
    "avd_engine_create": (C.c_int, [_P(AvdEngineSpec), _P(AvdTuning), _P(_E)]),
    "avd_engine_destroy": (None, [_E]),
    "avd_engine_set_stream": (C.c_int, [_E, C.c_void_p]),
    "avd_engine_push": (C.c_int, [_E, _P(AvdPlane), C.c_size_t, _P(C.c_size_t)]),
    "avd_engine_push_context": (C.c_int, [_E, _P(AvdPlane), C.c_size_t]),
    "avd_engine_emit_into": (C.c_int, [_E, _P(AvdPlane), C.c_size_t]),
    "avd_engine_finish": (C.c_int, [_E, _P(C.c_size_t)]),
    "avd_engine_reset": (C.c_int, [_E]),
    "avd_engine_window_span": (C.c_int, [_E, _P(AvdWindowSpan)]),
    "avd_engine_max_held_frames": (C.c_int, [_E, _P(C.c_size_t)]),
    "avd_engine_timing": (C.c_int, [_E, _P(AvdPassTimings)]),
    "avd_engine_sample_device_time": (C.c_int, [_E, u32]),
    "avd_engine_last_error": (C.c_char_p, [_E]),
    "avd_engine_fail_for_test": (C.c_int, [_E]),
    "avd_last_error": (C.c_char_p, []),
    "avd_host_create": (C.c_int, [_P(AvdEngineSpec), _P(AvdTuning), _P(_H)]),
    "avd_host_destroy": (None, [_H]),
    "avd_host_plane_bytes": (u64, [_H, C.c_size_t]),
    "avd_host_push": (C.c_int, [_H, _P(C.c_void_p), _P(u64), C.c_size_t]),
    "avd_host_push_priming": (C.c_int, [_H, _P(C.c_void_p), _P(u64), C.c_size_t]),
    "avd_host_recv": (C.c_int, [_H, _P(C.c_void_p), C.c_size_t, _P(C.c_int)]),
    "avd_host_flush": (C.c_int, [_H, AvdHostSink, C.c_void_p]),
    "avd_host_reset": (None, [_H]),
    "avd_host_last_error": (C.c_char_p, [_H]),
    "avd_host_poison_for_test": (None, [_H]),
    "avd_host_timing": (C.c_int, [_H, _P(AvdHostTiming)]),
    "avd_host_sample_device_time": (None, [_H, u32]),
    "avd_collab_pass": (C.c_int, [_P(AvdCollabPass), C.c_void_p]),
    "avd_collab_member_bytes": (u64, [u32, u32]),
    "avd_collab_refs": (u64, [u32, u32]),
    "avd_batch_ingest_scratch_bytes": (u64, [C.c_size_t]),
    "avd_batch_ingest": (C.c_int, [_P(AvdBatchIngest), C.c_size_t, u64, C.c_void_p]),
    "avd_collab_adjoint": (C.c_int, [_P(AvdCollabPass), _P(AvdCollabAdjoint), C.c_void_p]),
    "avd_dct_noise_profile": (None, [f32, _P(f32)]),
    "avd_kaiser_window": (None, [f32, _P(f32)]),
    "avd_cross_frame_accum_scale": (f32, [u32, u32]),
    "avd_motion_pyramid_floats": (u64, [u32, u32, u32, u32]),
    "avd_motion_pyramid_build": (C.c_int, [u64, u32, u32, u32, u32, u32, u32, u64, u32, C.c_void_p]),
    "avd_motion_search": (C.c_int, [_P(AvdMotionPass), C.c_void_p]),
    "avd_truemotion_pass": (C.c_int, [_P(AvdTruemotionPass), C.c_void_p]),
    "avd_escalation_state_floats": (u64, [u32, u32]),
    "avd_engine_models": (C.c_int, [_E, _P(f32), u32, _P(u32)]),
    "avd_model_fit_scratch_floats": (u64, [u32]),
    "avd_model_fit": (C.c_int, [_P(AvdModelFit), C.c_void_p]),
    "avd_compose_models": (C.c_int, [u64, u64, u64, u32, u32, u32, C.c_void_p]),
    "avd_block_means": (C.c_int, [u64, u64, u32, u32, u32, u32, C.c_void_p]),
    "avd_high_pass": (C.c_int, [u64, u64, u64, u32, u32, u32, C.c_void_p]),
    "avd_chain_compose": (C.c_int, [u64, u64, u32, u32, u32, u32, u32, u32, u32, u32, u32, C.c_void_p]),
    "avd_sad_noise_floor": (f32, [u32, f32]),
    "avd_thsad": (f32, [u32, f32]),
    "avd_immerkaer_partials_len": (u64, [u32, u32]),
    "avd_immerkaer": (C.c_int, [u64, u32, u32, u32, u64, u64, u64, C.c_void_p]),
    "avd_noise_records_floats": (u64, [u32, u32, u32]),
    "avd_noise_scratch_floats": (u64, [u32, u32]),
    "avd_noise_temporal_stats": (C.c_int, [u64, u64, u32, u32, u32, u32, u64, C.c_void_p]),
    "avd_noise_compensated_stats": (C.c_int, [u64, u64, u32, u32, u32, u64, u32, u32, u32, u32, u64, C.c_void_p]),
    "avd_noise_reading": (C.c_int, [u64, u32, u32, u32, u32, u64, u64, C.c_void_p]),
    "avd_colour_records": (u64, [u32, u32]),
    "avd_tune_variant_for_test": (C.c_int, [u32, C.c_char_p, C.c_char_p, u32, C.POINTER(C.c_float)]),
    "avd_tune_forget": (None, []),
    "avd_colour_means": (C.c_int, [u64, u64, u64, C.POINTER(AvdGeometry), u64, u64, C.c_void_p]),
    "avd_colour_accumulate": (C.c_int, [u64, u64, u32, u32, u32, u32, C.c_float, u64, C.c_void_p]),
    "avd_colour_window": (C.c_int, [u64, u32, u32, u32, u32, u64, C.c_void_p]),
    "avd_colour_fit_scratch_floats": (u64, [u32]),
    "avd_colour_fit": (C.c_int, [u64, u32, u32, u64, u64, u64, u64, u64, C.c_void_p]),
    "avd_colour_lookup": (C.c_int, [u64, u64, u32, u64, u64, C.c_void_p]),
    "avd_noise_fold_words": (None, [u32, u32, f32, u32, f32, f32, u32, f32, f32, f32, f32, u32, f32, f32, _P(f32)]),
    "avd_noise_fold": (C.c_int, [u64, u64, u32, u32, u32, u64, u32, u32, u64, u64, u64, u64, C.c_void_p]),
    "avd_nlm_backward_scratch_bytes": (u64, [u32, u32]),
    "avd_nlm_backward": (C.c_int, [_P(AvdNlmBackward), C.c_void_p]),
    "avd_nlm_window_scratch_bytes": (u64, [u32]),
    "avd_nlm_window": (C.c_int, [_P(AvdNlmBackward), C.c_void_p]),
    "avd_exp_mirror": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p]),
    "avd_batch_scratch_bytes": (u64, [C.c_size_t, u32]),
    "avd_batch_submit": (C.c_int, [_P(AvdBatchJob), C.c_size_t, u32, u32, u32, f32, u64, C.c_void_p]),
    "avd_nlm_frame_static": (C.c_int, [_P(AvdNlmeansAlgorithm), u32, u32, u32, AvdSampleFormat, AvdSampleFormat,
                                       _P(AvdPlane), C.c_size_t, _P(AvdPlane), C.c_size_t, C.c_void_p]),
}

_lib: C.CDLL | None = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libavd_b200.so and binds every prototype; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"libavd_b200.so is not built ({p}); run `python av-denoise_b200/build.py` or "
            "`__graft_entry__.build()` first. There is no CPU fallback."
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
