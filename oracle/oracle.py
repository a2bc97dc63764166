"""CPU ORACLE - test infrastructure only (see nlm_oracle.cpp). Loaded by tests/, by
`__graft_entry__.smoke()` and by the CPU-baseline leg of bench.py, as the checker; the product
never imports it.

ctypes bindings to liboracle.so plus the stream-level restatement of the NLMeans engine with
repeat edges (av-denoise-core/src/nlmeans/denoiser/ring.rs:103-146): output frame n is the
windowed NLM of frames clamp(n + k, 0, N - 1), k in -d..=d.
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_lib = None
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_fpp = C.POINTER(_fp)
_u32p = C.POINTER(C.c_uint32)


def build() -> Path:
    """Builds liboracle.so with its Makefile (gcc, -ffp-contract=off)."""
    res = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        l = C.CDLL(str(LIB))
        l.orc_ingest_words.argtypes = [_u32p, _u32p, _fp, C.c_int64, C.c_int, C.c_int, C.c_float]
        l.orc_ingest_f32.argtypes = [_fp, _fp, _fp, C.c_int64, C.c_int, C.c_float]
        l.orc_egress_words.argtypes = [_fp, _u32p, _u32p, C.c_int64, C.c_int, C.c_int, C.c_float]
        l.orc_egress_f32.argtypes = [_fp, _fp, _fp, C.c_int64, C.c_int, C.c_float]
        l.orc_h2_inv_norm.argtypes = [C.c_float, C.c_int]
        l.orc_h2_inv_norm.restype = C.c_float
        l.orc_welsch_weight.argtypes = [C.c_float, C.c_float, C.c_float]
        l.orc_welsch_weight.restype = C.c_float
        l.orc_exp_mirror.argtypes = [_fp, _fp, C.c_int64]
        l.orc_nlm_frame_f32.argtypes = [_fpp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                        C.c_float, _fp, _fpp, _fpp, C.c_int, C.c_int, C.c_int, C.c_float, _fp]
        l.orc_nlm_frame_f64.argtypes = [_fpp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                        C.c_double, _fp, _fpp, _fpp, C.c_int, C.c_int, C.c_int, C.c_double, _dp]
        l.orc_nlm_frame_ref_f32.argtypes = [_fpp, _fpp] + l.orc_nlm_frame_f32.argtypes[1:]
        l.orc_nlm_frame_ref_f64.argtypes = [_fpp, _fpp] + l.orc_nlm_frame_f64.argtypes[1:]
        l.orc_bilateral_f32.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _fp]
        _lib = l
    return _lib


def _f(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def h2_inv_norm(strength: float, patch_radius: int) -> float:
    return float(lib().orc_h2_inv_norm(strength, patch_radius))


def welsch_weight(total: float, h2: float, offset: float) -> float:
    return float(lib().orc_welsch_weight(total, h2, offset))


def exp_mirror(x: np.ndarray) -> np.ndarray:
    """The FP32 mirror's exponential (nlm_oracle.cpp `exp_mirror`) over a float32 array."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_exp_mirror(_f(x), _f(out), x.size)
    return out


def words_from_codes(codes: np.ndarray, fmt_kind: int) -> np.ndarray:
    """Packs a plane of integer codes into little-endian 32-bit words (u8: 4 per word, u16: 2)."""
    flat = codes.reshape(-1)
    if fmt_kind == 0:
        pad = (-flat.size) % 4
        b = np.concatenate([flat.astype(np.uint8), np.zeros(pad, np.uint8)])
    else:
        pad = (-flat.size) % 2
        b = np.concatenate([flat.astype(np.uint16), np.zeros(pad, np.uint16)])
    return np.ascontiguousarray(b).view(np.uint32)


def ingest(planes: list[np.ndarray], fmt_kind: int, max_value: float, bias: float = 0.0) -> np.ndarray:
    """Planes (codes, or f32 for kind 2) -> one interleaved normalised f32 frame (H, W, C)."""
    h, w = planes[0].shape
    c = len(planes)
    out = np.empty((h, w, c), np.float32)
    if fmt_kind == 2:
        p0 = np.ascontiguousarray(planes[0], np.float32)
        p1 = np.ascontiguousarray(planes[-1], np.float32)
        lib().orc_ingest_f32(_f(p0), _f(p1), _f(out), h * w, c, bias)
        return out
    w0 = words_from_codes(planes[0], fmt_kind)
    w1 = words_from_codes(planes[-1], fmt_kind)
    spw = 4 if fmt_kind == 0 else 2
    lib().orc_ingest_words(w0.ctypes.data_as(_u32p), w1.ctypes.data_as(_u32p), _f(out), h * w, c, spw, max_value)
    return out


def egress(frame: np.ndarray, fmt_kind: int, max_value: float, bias: float = 0.0) -> list[np.ndarray]:
    """Interleaved f32 frame (H, W, C) -> planes of codes (or f32 for kind 2)."""
    h, w, c = frame.shape
    fr = np.ascontiguousarray(frame, np.float32)
    if fmt_kind == 2:
        p = [np.empty((h, w), np.float32) for _ in range(2)]
        lib().orc_egress_f32(_f(fr), _f(p[0]), _f(p[1]), h * w, c, bias)
        return p[:c]
    spw = 4 if fmt_kind == 0 else 2
    words = (h * w + spw - 1) // spw
    p = [np.zeros(words, np.uint32) for _ in range(2)]
    lib().orc_egress_words(_f(fr), p[0].ctypes.data_as(_u32p), p[1].ctypes.data_as(_u32p), h * w, c, spw, max_value)
    dt = np.uint8 if fmt_kind == 0 else np.uint16
    return [q.view(dt)[: h * w].reshape(h, w).copy() for q in p[:c]]


def nlm_frame(window: list[np.ndarray], d: int, a: int, s: int, h2: float, noise_offset: float = 0.0,
              lut: np.ndarray | None = None, conf: list[tuple[np.ndarray, np.ndarray]] | None = None,
              conf_step: int = 8, blocks: tuple[int, int] = (1, 1), wref: float = 1.0,
              fp64: bool = False, refs: list[np.ndarray] | None = None) -> np.ndarray:
    """One windowed NLM output frame (FP32 mirror, or FP64). `window` holds 2d+1 (H, W, C) f32
    frames, the centre at index d; `refs`, when given, the prefilter's reference frames of the same
    window, which the patch distances compare instead."""
    assert len(window) == 2 * d + 1
    h, w, c = window[0].shape
    frames = [np.ascontiguousarray(f, np.float32) for f in window]
    arr = (_fp * len(frames))(*[_f(f) for f in frames])
    rframes = [np.ascontiguousarray(f, np.float32) for f in refs] if refs is not None else None
    rarr = (_fp * len(rframes))(*[_f(f) for f in rframes]) if rframes is not None else None
    lut_p = _f(np.ascontiguousarray(lut, np.float32)) if lut is not None else None
    cf = cb = None
    keep = []
    if conf:
        fw = [np.ascontiguousarray(x[0], np.float32) for x in conf]
        bw = [np.ascontiguousarray(x[1], np.float32) for x in conf]
        keep += fw + bw
        cf = (_fp * d)(*[_f(x) for x in fw])
        cb = (_fp * d)(*[_f(x) for x in bw])
    if fp64:
        out = np.empty((h, w, c), np.float64)
        lib().orc_nlm_frame_ref_f64(arr, rarr, w, h, c, d, a, s, h2, noise_offset, lut_p, cf, cb, conf_step,
                                    blocks[0], blocks[1], wref, out.ctypes.data_as(_dp))
    else:
        out = np.empty((h, w, c), np.float32)
        lib().orc_nlm_frame_ref_f32(arr, rarr, w, h, c, d, a, s, h2, noise_offset, lut_p, cf, cb, conf_step,
                                    blocks[0], blocks[1], wref, _f(out))
    return out


def bilateral_radius(sigma_s: float) -> int:
    """nlmeans/prefilter/bilateral.rs:11-13: max(ceil(2 sigma_s), 1), in f32."""
    return max(int(np.ceil(np.float32(2.0) * np.float32(sigma_s))), 1)


def inv_two_sigma_sq(sigma: float) -> float:
    """nlmeans/prefilter/bilateral.rs:20-22: 1 / (2 sigma^2), in f32."""
    f = np.float32
    return float(f(1.0) / ((f(2.0) * f(sigma)) * f(sigma)))


def bilateral(frame: np.ndarray, sigma_s: float, sigma_r: float) -> np.ndarray:
    """The bilateral prefilter of one (H, W, C) f32 frame (nlmeans/kernels/bilateral.rs:16-107)."""
    h, w, c = frame.shape
    src = np.ascontiguousarray(frame, np.float32)
    out = np.empty_like(src)
    lib().orc_bilateral_f32(_f(src), w, h, c, bilateral_radius(sigma_s), inv_two_sigma_sq(sigma_s),
                            inv_two_sigma_sq(sigma_r), _f(out))
    return out


def pilot_h2(h2: float, strength_scale: float) -> float:
    """nlmeans/dispatch/mod.rs:40-43: h2 / strength_scale^2, in f32."""
    f = np.float32
    return float(f(h2) / (f(strength_scale) * f(strength_scale)))


def flat_offset_lut(a: int, offset: float) -> np.ndarray:
    """noise/correlation.rs:71-88 at rho 0: `offset` for every candidate but the centre."""
    side = 2 * a + 1
    lut = np.full(side * side, offset, np.float32)
    lut[a * side + a] = 0.0
    return lut


def prefilter_refs(frames: list[np.ndarray], prefilter, a: int, s: int, wref: float = 1.0) -> list[np.ndarray]:
    """The reference frame of every stream frame under a fixed-strength prefilter
    (nlmeans/denoiser/stages.rs:29-59): ("bilateral", sigma_s, sigma_r) blurs each frame;
    ("nlm", pilot_h2, pilot_lut) denoises each frame alone with the windowed spatial pass at the
    pilot strength and offset table (dispatch/mod.rs:598-620). The references are a function of
    their own frame only, so an edge duplicate's reference is its frame's."""
    kind = prefilter[0]
    if kind == "bilateral":
        return [bilateral(f, prefilter[1], prefilter[2]) for f in frames]
    assert kind == "nlm"
    return [nlm_frame([f], 0, a, s, prefilter[1], lut=prefilter[2], wref=wref) for f in frames]


def nlm_stream_repeat(frames: list[np.ndarray], d: int, a: int, s: int, h2: float, wref: float = 1.0,
                      noise_offset: float = 0.0, fp64: bool = False, lut: np.ndarray | None = None,
                      conf_sigma: float | None = None, thsad_scale: float = 1.0, prefilter=None) -> list[np.ndarray]:
    """The NLMeans engine over a whole stream with repeat edges: one output per input. With
    `conf_sigma`, every temporal weight is scaled by the HQ confidence pass at that pinned sigma.
    With `prefilter` (see `prefilter_refs`) the distances compare the reference frames; the
    references themselves are always the FP32 mirror's, as the engine keeps them in f32."""
    n = len(frames)
    refs = prefilter_refs(frames, prefilter, a, s, wref) if prefilter is not None else None
    outs = []
    for i in range(n):
        idx = [min(max(i + k, 0), n - 1) for k in range(-d, d + 1)]
        window = [frames[j] for j in idx]
        conf, blocks = None, (1, 1)
        if conf_sigma is not None and d > 0:
            conf, blocks = hq_confidence(window, d, conf_sigma, thsad_scale)
        outs.append(nlm_frame(window, d, a, s, h2, noise_offset=noise_offset, lut=lut, conf=conf, conf_step=8,
                              blocks=blocks, wref=wref, fp64=fp64,
                              refs=[refs[j] for j in idx] if refs is not None else None))
    return outs


def mc_warp(frame: np.ndarray, mv: np.ndarray, step: int, bx: int, by: int) -> np.ndarray:
    """motion/kernels/compensate.rs:6-44 (`mc_warp`): pixel (x, y) takes the vector of block
    (min(x / step, bx - 1), min(y / step, by - 1)) and copies the source pixel at the clamped
    (x + dx, y + dy)."""
    h, w, _ = frame.shape
    ys, xs = np.mgrid[0:h, 0:w]
    v = np.asarray(mv, np.int32).reshape(by, bx, 2)[np.minimum(ys // step, by - 1), np.minimum(xs // step, bx - 1)]
    return frame[np.clip(ys + v[..., 1], 0, h - 1), np.clip(xs + v[..., 0], 0, w - 1)]


def nlm_stream_mc(frames: list[np.ndarray], d: int, a: int, s: int, h2: float, *, wref: float = 1.0,
                  noise_offset: float = 0.0, lut: np.ndarray | None = None, confidence: bool = False,
                  sad_floor: float = 0.0, thsad_scale: float = 1.0, blksize: int = 16, overlap: int = 8,
                  search_radius: int = 4, levels: int = 2, chained: bool = False, refine_radius: int = 2,
                  prefilter=None, fp64: bool = False, derived=None, share_writes=None,
                  share_reads=None, ceiling: int = 0, camera_model: bool = True,
                  models: "PairModels | None" = None) -> list[np.ndarray]:
    """NLMeans with motion compensation over a stream with repeat edges, replayed slot by slot as
    the ring runs it (nlmeans/denoiser/ring.rs, stages.rs:62-209, dispatch/motion.rs:104-487):
      - each slot write (and each edge copy) builds the slot's pyramids; with Chained estimation it
        then searches the pair between the slot and the one before it both ways (each direction
        ending with the truemotion stage, floor unread) into pair slot ring_head mod 2d, or zeroes
        that pair slot for an edge copy;
      - each window matches every neighbour against the centre on the reference's pyramid under a
        prefilter, else the input's: Chained walks the pair ring and refines `refine_radius` around
        the walk, Direct searches with its truemotion stage reading the window's floor; with
        `confidence` (HQ temporal confidence) the search scores each block against `sad_floor`;
      - every neighbour (and its reference) is warped along its field, the temporal passes compare
        the warped frames, weighted by the confidence of their motion blocks.
    `prefilter` is as in `prefilter_refs` (fixed strength). With `derived`, a function of a window's
    centre stream frame returning (h2, noise_offset, lut, sad_floor) (the automatic estimate's fold
    around that frame), each window reads those instead. `share_writes` / `share_reads` (a
    `MotionShare`) share each window's field with a chroma pass, or take the luma pass's mapped field
    and search one pixel around it at one level, as in `nl4d_stream`. With `camera_model` (the
    engine's default, engine/spec.rs:426-450) a pass that searches its own motion also searches
    around the camera models fitted on channel 0 of the frames (`models`, else a `PairModels` fed
    every frame in order): the Direct window search around each neighbour's composed prediction,
    the Chained pair searches around the pair's prediction with zeroed noise words. Returns one output
    per input."""
    n = len(frames)
    h, w, c = frames[0].shape
    tf = 2 * d + 1
    step = blksize - overlap
    bx, by = max(-(-w // step), 1), max(-(-h // step), 1)
    refs_of = prefilter_refs(frames, prefilter, a, s, wref) if prefilter is not None else None
    th = thsad(blksize, thsad_scale)
    slot_frame = [0] * tf
    zero = np.zeros((bx * by, 2), np.int32)
    pairs = {i: (zero, zero) for i in range(2 * d)}
    st = dict(head=0, loaded=0, call=0)
    if share_reads is not None:
        chained, levels = False, 1
    if camera_model and share_reads is None and models is None and d > 0:
        models = pair_models_for([f[..., 0] for f in frames], w, h, blksize=blksize, overlap=overlap,
                                 search_radius=search_radius, levels=levels, ceiling=ceiling)
    if not camera_model or share_reads is not None:
        models = None
    outs = []

    def search_pyramid():
        src = refs_of if refs_of is not None else frames
        ring = np.stack([src[f] for f in slot_frame]).astype(np.float32)
        return motion_pyramid(ring.reshape(-1), c, w, h, levels)

    def write(slot, frame_idx, duplicate):
        slot_frame[slot] = frame_idx
        if not chained:
            return
        if duplicate:
            pairs[st["head"] % (2 * d)] = (zero, zero)
        elif st["head"] > 0:
            older = (slot + tf - 1) % tf
            pyr = search_pyramid()
            kw = dict(blksize=blksize, overlap=overlap, search_radius=search_radius, levels=levels, thsad=th,
                      field_lambda=1.0, reads_floor=False, ceiling=ceiling)
            o2n, n2o = models.compose_pair(slot_frame[older], frame_idx) if models is not None else (None, None)
            fwd, _ = motion_search(pyr, w, h, tf, older, [slot], predictions=o2n, **kw)
            bwd, _ = motion_search(pyr, w, h, tf, slot, [older], predictions=n2o, **kw)
            pairs[st["head"] % (2 * d)] = (fwd[0], bwd[0])

    def duplicate_last():
        last, nxt = (st["head"] - 1) % tf, st["head"] % tf
        write(nxt, slot_frame[last], True)
        st["head"] += 1

    def enter(frame_idx):
        write(st["head"] % tf, frame_idx, False)
        st["head"] += 1
        st["loaded"] = min(st["loaded"] + 1, tf)
        if st["loaded"] == 1:
            for _ in range(d):
                duplicate_last()
                st["loaded"] += 1

    def denoise():
        if st["loaded"] < tf:
            return
        phys = [(st["head"] % tf + l) % tf for l in range(tf)]
        cs = phys[d]
        slots = [phys[l] for l in range(tf) if l != d]
        w_h2, w_off, w_lut, w_floor = h2, noise_offset, lut, sad_floor
        if derived is not None:
            w_h2, w_off, w_lut, w_floor = derived(slot_frame[cs])
        pyr = search_pyramid()
        if share_reads is not None:
            mapped = share_reads.read(st["call"], slot_frame[cs] % tf, slot_frame[cs])
            mv, cf = motion_search(pyr, w, h, tf, cs, slots, blksize=blksize, overlap=overlap, search_radius=1,
                                   levels=1, confidence=confidence, sad_floor=w_floor, thsad=th, seeds=mapped)
        elif chained:
            seeds = chain_compose(pairs, d, d, st["head"] % (2 * d), step, w, h, bx, by)
            mv, cf = motion_search(pyr, w, h, tf, cs, slots, blksize=blksize, overlap=overlap,
                                   search_radius=refine_radius, levels=levels, confidence=confidence,
                                   sad_floor=w_floor, thsad=th, seeds=seeds, ceiling=ceiling, esc_reads_floor=True)
        else:
            pred = models.compose_window([slot_frame[p] for p in phys], d) if models is not None else None
            mv, cf = motion_search(pyr, w, h, tf, cs, slots, blksize=blksize, overlap=overlap,
                                   search_radius=search_radius, levels=levels, confidence=confidence,
                                   sad_floor=w_floor, thsad=th, field_lambda=1.0, reads_floor=True, ceiling=ceiling,
                                   esc_reads_floor=True, predictions=pred)
        if share_writes is not None:
            share_writes.write(st["call"], slot_frame[cs] % tf, slot_frame[cs], mv)
        window, refs = [], []
        idx = 0
        for l in range(tf):
            f = slot_frame[phys[l]]
            if l == d:
                window.append(frames[f])
                refs.append(refs_of[f] if refs_of is not None else None)
                continue
            window.append(mc_warp(frames[f], mv[idx], step, bx, by))
            refs.append(mc_warp(refs_of[f], mv[idx], step, bx, by) if refs_of is not None else None)
            idx += 1
        conf = [(cf[k], cf[2 * d - 1 - k]) for k in range(d)] if confidence else None
        outs.append(nlm_frame(window, d, a, s, w_h2, noise_offset=w_off, lut=w_lut, conf=conf, conf_step=step,
                              blocks=(bx, by), wref=wref, fp64=fp64,
                              refs=refs if refs_of is not None else None))

    for i in range(n):
        st["call"] = i
        enter(i)
        denoise()
    while len(outs) < n:
        st["call"] = n + len(outs)
        duplicate_last()
        st["loaded"] = min(st["loaded"] + 1, tf)
        denoise()
    return outs


def hq_confidence(window: list[np.ndarray], d: int, sigma: float, thsad_scale: float = 1.0,
                  sad_floor: float | None = None):
    """The HQ confidence pass over one window (nlmeans/dispatch/motion.rs:554-613): lane 0 of every
    frame, 16x16 blocks at step 8 scored where they stand against the centre, floor
    sad_noise_floor(16, sigma), thsad(16, thsad_scale). Returns the (forward, backward) block
    confidences of each pair k (q_k = -d + k) and the block grid."""
    h, w, c = window[0].shape
    ring = np.stack([np.ascontiguousarray(f, np.float32) for f in window]).reshape(-1)
    pyr = motion_pyramid(ring, c, w, h, 1)
    slots = [l for l in range(2 * d + 1) if l != d]
    _, conf = motion_search(pyr, w, h, 2 * d + 1, d, slots, blksize=16, overlap=8, search_radius=0, levels=1,
                            confidence=True, sad_floor=sad_noise_floor(16, sigma) if sad_floor is None else sad_floor,
                            thsad=thsad(16, thsad_scale))
    blocks = (max(-(-w // 8), 1), max(-(-h // 8), 1))
    return [(conf[k], conf[2 * d - 1 - k]) for k in range(d)], blocks


# ---- NL4D collaborative filter (collab_oracle.cpp) ------------------------------------------------

class CollabArgs(C.Structure):
    _fields_ = [
        ("ring", _fp), ("mv_field", C.POINTER(C.c_int32)), ("confidence", _fp),
        ("neighbour_slots", C.POINTER(C.c_uint32)), ("sigma", _fp), ("noise_curve", _fp),
        ("dct_profile", _fp), ("kaiser", _fp), ("accum", C.POINTER(C.c_int32)),
        ("wsum", C.POINTER(C.c_int32)), ("group_weight", _fp),
        ("width", C.c_int), ("height", C.c_int), ("channels", C.c_int), ("centre_slot", C.c_int),
        ("radius", C.c_int), ("grid_frames", C.c_int), ("refine", C.c_int), ("spatial_radius", C.c_int),
        ("k_max", C.c_int), ("mv_stride", C.c_int), ("conf_stride", C.c_int), ("blk_step", C.c_int),
        ("blksize", C.c_int), ("blocks_x", C.c_int), ("blocks_y", C.c_int),
        ("c_min", C.c_float), ("lambda_ht", C.c_float), ("accum_scale", C.c_float), ("pool_ratio", C.c_float),
        ("weight_scale", C.c_float), ("pooled", C.c_int), ("curve_valid", C.c_int),
        ("colour_gains", _fp), ("colour_means", _fp), ("colour_scale", C.c_float), ("colour_on", C.c_int),
        ("colour_blocks_x", C.c_int), ("wiener", C.c_int), ("member_record", _u32p),
        ("mask_record", C.POINTER(C.c_uint64)),
    ]


class Collab64Args(C.Structure):
    _fields_ = [
        ("ring", _dp), ("members", _u32p), ("masks", C.POINTER(C.c_uint64)), ("neighbour_slots", _u32p),
        ("sigma", _dp), ("dct_profile", _fp), ("kaiser", _fp), ("weight_scale", C.c_double),
        ("weight_scale_sigma", C.c_double),
        ("width", C.c_int), ("height", C.c_int), ("channels", C.c_int), ("centre_slot", C.c_int),
        ("grid_frames", C.c_int), ("wiener", C.c_int),
        ("accum", _dp), ("wsum", _dp), ("grad_accum", _dp), ("grad_wsum", _dp), ("grad_ring", _dp),
        ("grad_sigma", _dp),
    ]


def dct_noise_profile(rho: float) -> np.ndarray:
    out = np.empty(8, np.float32)
    l = lib()
    l.orc_dct_noise_profile.argtypes = [C.c_float, _fp]
    l.orc_dct_noise_profile(rho, _f(out))
    return out


def kaiser_window(beta: float) -> np.ndarray:
    out = np.empty(8, np.float32)
    l = lib()
    l.orc_kaiser_window.argtypes = [C.c_float, _fp]
    l.orc_kaiser_window(beta, _f(out))
    return out


def cross_frame_accum_scale(spatial_radius: int, temporal_radius: int) -> float:
    l = lib()
    l.orc_cross_frame_accum_scale.argtypes = [C.c_uint32, C.c_uint32]
    l.orc_cross_frame_accum_scale.restype = C.c_float
    return float(l.orc_cross_frame_accum_scale(spatial_radius, temporal_radius))


def weight_scale(sigma: float, profile: np.ndarray) -> float:
    """aggregate.rs:79-99: sigma^2 * g_max^2 in f32, floored at 1e-12."""
    f = np.float32
    g = f(np.max(profile))
    norm = ((f(sigma) * f(sigma)) * g) * g
    return float(norm) if np.isfinite(norm) and norm > f(1e-12) else 1e-12


def grid_frames(radius: int) -> int:
    """collab/mod.rs:48-54."""
    return 1 if radius == 0 else (2 if radius == 1 else 4)


def refs_along(dim: int) -> int:
    return (dim - 8 + 3) // 4 + 1


def collab_fused(ring: np.ndarray, width: int, height: int, channels: int, *, centre_slot=0, radius=0,
                 mv_field=None, confidence=None, neighbour_slots=None, c_min=0.0, refine=0, spatial_radius=4,
                 k_max=8, sigma=(0.02,), lambda_ht=5.3, rho=0.0, profile=None, kaiser_beta=0.0,
                 noise_curve=None, pooled=None, blksize=16, blk_step=8, blocks_x=1, blocks_y=1,
                 mv_stride=2, conf_stride=1, weight_scale_override=None, colour=None, wiener=False,
                 record=None):
    """One `collab_fused` launch on the CPU. Returns (accum, wsum, group_weight). `colour` is
    (gains tables, block means on this plane's 16x16 grid, 8-bit scale) or None. `wiener` adds the
    empirical Wiener stage. A dict passed as `record` receives the pass's member words ("members",
    9 u32 per reference patch) and keep masks ("masks", refs x channels x 8 u64)."""
    ring = np.ascontiguousarray(ring, np.float32)
    frames = ring.size // (width * height * channels)
    profile = dct_noise_profile(rho) if profile is None else np.asarray(profile, np.float32)
    kaiser = kaiser_window(kaiser_beta)
    sig = np.asarray(sigma, np.float32)
    if sig.size < channels:
        sig = np.full(channels, sig[0], np.float32)
    ws = weight_scale(float(sig[0]), profile) if weight_scale_override is None else weight_scale_override
    mv = np.ascontiguousarray(mv_field if mv_field is not None else np.zeros(2, np.int32), np.int32)
    conf = np.ascontiguousarray(confidence if confidence is not None else np.ones(1, np.float32), np.float32)
    slots = np.ascontiguousarray(neighbour_slots if neighbour_slots is not None else np.zeros(1, np.uint32),
                                 np.uint32)
    curve = np.ascontiguousarray(noise_curve if noise_curve is not None else np.zeros(16, np.float32), np.float32)
    accum = np.zeros(width * height * channels * frames, np.int32)
    wsum = np.zeros(width * height * frames, np.int32)
    gw = np.zeros(refs_along(width) * refs_along(height), np.float32)
    a = CollabArgs()
    a.ring, a.mv_field, a.confidence = _f(ring), mv.ctypes.data_as(C.POINTER(C.c_int32)), _f(conf)
    a.neighbour_slots = slots.ctypes.data_as(C.POINTER(C.c_uint32))
    a.sigma, a.noise_curve, a.dct_profile, a.kaiser = _f(sig), _f(curve), _f(profile), _f(kaiser)
    a.accum, a.wsum = accum.ctypes.data_as(C.POINTER(C.c_int32)), wsum.ctypes.data_as(C.POINTER(C.c_int32))
    a.group_weight = _f(gw)
    a.width, a.height, a.channels, a.centre_slot = width, height, channels, centre_slot
    a.radius, a.grid_frames, a.refine, a.spatial_radius, a.k_max = radius, grid_frames(radius), refine, \
        spatial_radius, k_max
    a.mv_stride, a.conf_stride, a.blk_step, a.blksize = mv_stride, conf_stride, blk_step, blksize
    a.blocks_x, a.blocks_y = blocks_x, blocks_y
    a.c_min, a.lambda_ht = c_min, lambda_ht
    a.accum_scale = cross_frame_accum_scale(spatial_radius, radius)
    a.pool_ratio, a.pooled = (pooled or 0.0), int(pooled is not None)
    a.weight_scale, a.curve_valid = ws, int(noise_curve is not None)
    if colour is not None:
        cg = np.ascontiguousarray(colour[0], np.float32)
        cm = np.ascontiguousarray(colour[1], np.float32).reshape(-1)
        a.colour_gains, a.colour_means, a.colour_scale = _f(cg), _f(cm), float(colour[2])
        a.colour_on, a.colour_blocks_x = 1, -(-width // 16)
    a.wiener = int(bool(wiener))
    refs = refs_along(width) * refs_along(height)
    if record is not None:
        record["members"] = np.zeros(refs * 9, np.uint32)
        record["masks"] = np.zeros(refs * channels * 8, np.uint64)
        a.member_record = record["members"].ctypes.data_as(_u32p)
        a.mask_record = record["masks"].ctypes.data_as(C.POINTER(C.c_uint64))
        record["weight_scale"] = ws
        record["sigma"] = sig
        record["profile"] = profile
        record["kaiser"] = kaiser
    l = lib()
    l.orc_collab_fused.argtypes = [C.POINTER(CollabArgs)]
    l.orc_collab_fused(C.byref(a))
    return accum, wsum, gw


def collab64(ring: np.ndarray, width: int, height: int, channels: int, record: dict, *, centre_slot=0, radius=0,
             neighbour_slots=None, sigma=None, wiener=False, grad_accum=None, grad_wsum=None):
    """The f64 pass of collab_adjoint_oracle.cpp over the groups and keep masks of `record` (from
    `collab_fused(..., record=...)`). Without gradients returns (accum, wsum) in real units; with
    `grad_accum` and `grad_wsum` returns (grad_ring, grad_sigma). `sigma` (per channel, f64)
    defaults to the recorded pass's."""
    ring = np.ascontiguousarray(ring, np.float64)
    frames = ring.size // (width * height * channels)
    sig = np.ascontiguousarray(record["sigma"] if sigma is None else sigma, np.float64)
    if sig.size < channels:
        sig = np.full(channels, sig[0], np.float64)
    slots = np.ascontiguousarray(neighbour_slots if neighbour_slots is not None else np.zeros(1, np.uint32),
                                 np.uint32)
    prof = np.ascontiguousarray(record["profile"], np.float32)
    kai = np.ascontiguousarray(record["kaiser"], np.float32)
    a = Collab64Args()
    a.ring, a.members = ring.ctypes.data_as(_dp), record["members"].ctypes.data_as(_u32p)
    a.masks = record["masks"].ctypes.data_as(C.POINTER(C.c_uint64))
    a.neighbour_slots, a.sigma = slots.ctypes.data_as(_u32p), sig.ctypes.data_as(_dp)
    a.dct_profile, a.kaiser, a.weight_scale = _f(prof), _f(kai), float(record["weight_scale"])
    a.weight_scale_sigma = float(np.float32(record["sigma"][0]))
    a.width, a.height, a.channels, a.centre_slot = width, height, channels, centre_slot
    a.grid_frames, a.wiener = grid_frames(radius), int(bool(wiener))
    l = lib()
    l.orc64_collab_pass.argtypes = [C.POINTER(Collab64Args)]
    if grad_accum is None:
        accum = np.zeros(width * height * channels * frames, np.float64)
        wsum = np.zeros(width * height * frames, np.float64)
        a.accum, a.wsum = accum.ctypes.data_as(_dp), wsum.ctypes.data_as(_dp)
        l.orc64_collab_pass(C.byref(a))
        return accum, wsum
    ga = np.ascontiguousarray(grad_accum, np.float64)
    gw = np.ascontiguousarray(grad_wsum, np.float64)
    grad_ring = np.zeros_like(ring)
    grad_sigma = np.zeros(channels, np.float64)
    a.grad_accum, a.grad_wsum = ga.ctypes.data_as(_dp), gw.ctypes.data_as(_dp)
    a.grad_ring, a.grad_sigma = grad_ring.ctypes.data_as(_dp), grad_sigma.ctypes.data_as(_dp)
    l.orc64_collab_pass(C.byref(a))
    return grad_ring, grad_sigma


# ---- block-matching motion search (motion_oracle.cpp) -------------------------------------------

class MotionArgs(C.Structure):
    _fields_ = [
        ("pyramid", _fp), ("neighbour_slots", C.POINTER(C.c_uint32)), ("mv_field", C.POINTER(C.c_int32)),
        ("confidence", _fp), ("noise", _fp),
    ] + [(n, C.c_uint32) for n in ("width", "height", "frame_count", "centre_slot", "neighbours", "blksize",
                                   "overlap", "search_radius", "levels", "mv_stride", "conf_stride",
                                   "sad_floor_word")] + [("thsad", C.c_float), ("seeded", C.c_uint32),
                                                         ("keep_seeds", C.POINTER(C.c_int32))] + \
        [(n, C.c_uint32) for n in ("ceiling", "esc_reads_floor", "widen_coarse")] + \
        [("predictions", _fp), ("sad_out", _fp), ("coarse_radius", C.c_uint32), ("coarse_block_factor", C.c_uint32)]


class TruemotionArgs(C.Structure):
    _fields_ = [
        ("pyramid", _fp), ("neighbour_slots", C.POINTER(C.c_uint32)), ("mv_in", C.POINTER(C.c_int32)),
        ("seeds", C.POINTER(C.c_int32)), ("mv_out", C.POINTER(C.c_int32)), ("confidence", _fp), ("noise", _fp),
    ] + [(n, C.c_uint32) for n in ("width", "height", "frame_count", "centre_slot", "neighbours", "blksize",
                                   "overlap", "mv_stride", "conf_stride", "sad_field", "reads_floor",
                                   "refine_radius")] + [(n, C.c_float) for n in ("lambda_base", "lambda_noise",
                                                                                 "surcharge", "fade_level", "thsad")] + \
        [("changes_in", C.POINTER(C.c_uint32)), ("changes_out", C.POINTER(C.c_uint32)),
         ("predictions", _fp), ("sad_out", _fp)]


# motion/truemotion/params.rs:4-33 and motion/confidence.rs:10.
TRUEMOTION = dict(noise_weight=1.0, surcharge=0.125, fade_scale=2.0, refine_radius=1)
THSAD_PIXEL = 0.02


def truemotion_values(field_lambda: float, blksize: int, thsad_value: float) -> tuple[float, float, float]:
    """motion/truemotion/stage.rs:52-62 in f32: (lambda_base, lambda_noise, fade_level)."""
    f = np.float32
    base = f(f(f(field_lambda) * f(blksize * blksize)) * f(THSAD_PIXEL))
    noise = f(f(field_lambda) * f(TRUEMOTION["noise_weight"]))
    fade = f(f(TRUEMOTION["fade_scale"]) * f(max(thsad_value, 0.0)))
    return float(base), float(noise), float(fade)


def truemotion_pass(pyramid: np.ndarray, width: int, height: int, frames: int, centre_slot: int, neighbour_slots,
                    mv_in: np.ndarray, seeds: np.ndarray | None, *, blksize=16, overlap=8, field_lambda=1.0,
                    thsad=0.0, sad_floor=0.0, reads_floor=True, confidence=False, passes=1, predictions=None,
                    sad_out: np.ndarray | None = None):
    """The truemotion stage: returns (mv (n, blocks, 2), conf (n, blocks)). With `passes` 2 (a search
    that escalates, truemotion/params.rs:9-12, 79-90) the second pass reads the first's field and
    rescores only the blocks next to one it changed (truemotion/stage.rs:82-142). With `predictions`
    (6 words per neighbour) the camera model's prediction is a candidate; with `sad_out` (f32, one per
    block per neighbour) every rescored block writes its winning SAD there."""
    mv = mv_in
    conf = None
    changes = None
    for p in range(passes):
        out_changes = np.zeros(np.asarray(mv_in).size // 2, np.uint32) if p + 1 < passes else None
        mv, c = _truemotion_once(pyramid, width, height, frames, centre_slot, neighbour_slots, mv, seeds,
                                 blksize=blksize, overlap=overlap, field_lambda=field_lambda, thsad=thsad,
                                 sad_floor=sad_floor, reads_floor=reads_floor, confidence=confidence,
                                 changes_in=changes, changes_out=out_changes, conf_in=conf, predictions=predictions,
                                 sad_out=sad_out)
        conf, changes = c, out_changes
    return mv, conf


def _truemotion_once(pyramid, width, height, frames, centre_slot, neighbour_slots, mv_in, seeds, *, blksize,
                     overlap, field_lambda, thsad, sad_floor, reads_floor, confidence, changes_in=None,
                     changes_out=None, conf_in=None, predictions=None, sad_out=None):
    step = blksize - overlap
    bx, by = max(-(-width // step), 1), max(-(-height // step), 1)
    slots = np.ascontiguousarray(neighbour_slots, np.uint32)
    n = slots.size
    mv_in = np.ascontiguousarray(mv_in, np.int32).reshape(-1)
    sd = np.ascontiguousarray(seeds, np.int32).reshape(-1) if seeds is not None else None
    out = np.zeros_like(mv_in)
    conf = np.zeros(n * bx * by, np.float32) if conf_in is None else np.ascontiguousarray(conf_in, np.float32).reshape(-1).copy()
    noise = np.array([sad_floor], np.float32)
    lb, ln, fade = truemotion_values(field_lambda, blksize, thsad)
    a = TruemotionArgs()
    a.pyramid, a.neighbour_slots = _f(pyramid), slots.ctypes.data_as(C.POINTER(C.c_uint32))
    a.mv_in = mv_in.ctypes.data_as(C.POINTER(C.c_int32))
    a.seeds = sd.ctypes.data_as(C.POINTER(C.c_int32)) if sd is not None else None
    a.mv_out = out.ctypes.data_as(C.POINTER(C.c_int32))
    a.confidence = _f(conf) if confidence else None
    a.noise = _f(noise)
    a.width, a.height, a.frame_count, a.centre_slot, a.neighbours = width, height, frames, centre_slot, n
    a.blksize, a.overlap, a.mv_stride, a.conf_stride = blksize, overlap, bx * by * 2, bx * by
    a.sad_field, a.reads_floor, a.refine_radius = 0, int(reads_floor), TRUEMOTION["refine_radius"]
    a.lambda_base, a.lambda_noise, a.surcharge, a.fade_level, a.thsad = lb, ln, TRUEMOTION["surcharge"], fade, thsad
    a.changes_in = changes_in.ctypes.data_as(C.POINTER(C.c_uint32)) if changes_in is not None else None
    a.changes_out = changes_out.ctypes.data_as(C.POINTER(C.c_uint32)) if changes_out is not None else None
    pred = np.ascontiguousarray(predictions, np.float32).reshape(-1) if predictions is not None else None
    a.predictions = _f(pred) if pred is not None else None
    a.sad_out = _f(sad_out) if sad_out is not None else None
    l = lib()
    l.orc_truemotion_pass.argtypes = [C.POINTER(TruemotionArgs)]
    l.orc_truemotion_pass(C.byref(a))
    return out.reshape(n, bx * by, 2), conf.reshape(n, bx * by)


def motion_pyramid(ring: np.ndarray, channels: int, width: int, height: int, levels: int) -> np.ndarray:
    """Every ring slot's luma pyramid, in the CUDA path's layout."""
    ring = np.ascontiguousarray(ring, np.float32)
    frames = ring.size // (width * height * channels)
    l = lib()
    l.orc_motion_pyramid_floats.argtypes = [C.c_int] * 4
    l.orc_motion_pyramid_floats.restype = C.c_int64
    pyr = np.zeros(l.orc_motion_pyramid_floats(width, height, frames, levels), np.float32)
    l.orc_motion_pyramid_build.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _fp, C.c_int]
    for slot in range(frames):
        l.orc_motion_pyramid_build(_f(ring), channels, width, height, frames, slot, levels, _f(pyr), slot)
    return pyr


def motion_search(pyramid: np.ndarray, width: int, height: int, frames: int, centre_slot: int, neighbour_slots,
                  *, blksize=16, overlap=8, search_radius=4, levels=2, confidence=False, sad_floor=0.0,
                  thsad=0.0, seeds: np.ndarray | None = None, field_lambda: float = 0.0, reads_floor: bool = True,
                  ceiling: int = 0, esc_reads_floor: bool = False, predictions=None, sad_out: np.ndarray | None = None,
                  coarse_radius: int | None = None, coarse_block_factor: int = 1):
    """One block-matching search. Returns (mv (n, blocks, 2), conf).
    With `predictions` (6 words per neighbour) every pass also searches around the neighbour's camera
    model prediction, that window winning by more than 1/8 of `sad_floor` (scaled to the coarse
    block on the coarse level). With `sad_out` (f32, 2 * n * blocks) the fine pass writes each
    block's winning SAD and then its window's mean SAD; the truemotion stage and the escalation
    replace the winning SAD. `coarse_radius` (default `search_radius`) and `coarse_block_factor` shape
    the coarse pass (motion/context.rs:99-105).
    With `seeds` (n, blocks, 2) the search refines around them and skips the coarse pass. With
    `ceiling` > `search_radius` the blocks that fail search again `ceiling` around their first
    window (motion/escalate.rs), the coarse level too when a coarse pass ran, and the truemotion
    stage runs two passes. With `field_lambda` > 0 the truemotion stage ends the search
    (motion/analyse.rs:175-312): its seed candidates are the coarse pass's field, when a coarse pass
    ran."""
    step = blksize - overlap
    bx, by = max(-(-width // step), 1), max(-(-height // step), 1)
    slots = np.ascontiguousarray(neighbour_slots, np.uint32)
    n = slots.size
    mv = np.zeros(n * bx * by * 2, np.int32) if seeds is None else np.ascontiguousarray(seeds, np.int32).reshape(-1).copy()
    conf = np.zeros(n * bx * by, np.float32)
    noise = np.array([sad_floor], np.float32)
    a = MotionArgs()
    a.pyramid, a.neighbour_slots = _f(pyramid), slots.ctypes.data_as(C.POINTER(C.c_uint32))
    a.mv_field = mv.ctypes.data_as(C.POINTER(C.c_int32))
    a.confidence = _f(conf) if confidence else None
    a.noise = _f(noise)
    a.width, a.height, a.frame_count, a.centre_slot, a.neighbours = width, height, frames, centre_slot, n
    a.blksize, a.overlap, a.search_radius, a.levels = blksize, overlap, search_radius, levels
    a.mv_stride, a.conf_stride, a.sad_floor_word, a.thsad = bx * by * 2, bx * by, 0, thsad
    a.seeded = int(seeds is not None)
    escalates = ceiling > search_radius
    a.ceiling, a.esc_reads_floor, a.widen_coarse = ceiling if escalates else 0, int(esc_reads_floor), 1
    coarse = levels > 1 and seeds is None
    kept = np.zeros_like(mv) if (field_lambda > 0.0 and coarse) else None
    a.keep_seeds = kept.ctypes.data_as(C.POINTER(C.c_int32)) if kept is not None else None
    pred = np.ascontiguousarray(predictions, np.float32).reshape(-1) if predictions is not None else None
    a.predictions = _f(pred) if pred is not None else None
    a.sad_out = _f(sad_out) if sad_out is not None else None
    a.coarse_radius = search_radius if coarse_radius is None else coarse_radius
    a.coarse_block_factor = coarse_block_factor
    l = lib()
    l.orc_motion_search.argtypes = [C.POINTER(MotionArgs)]
    l.orc_motion_search(C.byref(a))
    if field_lambda > 0.0:
        return truemotion_pass(pyramid, width, height, frames, centre_slot, slots, mv, kept, blksize=blksize,
                               overlap=overlap, field_lambda=field_lambda, thsad=thsad, sad_floor=sad_floor,
                               reads_floor=reads_floor, confidence=confidence, passes=2 if escalates else 1,
                               predictions=pred, sad_out=sad_out)
    return mv.reshape(n, bx * by, 2), conf.reshape(n, bx * by)


def sad_noise_floor(blksize: int, sigma: float) -> float:
    """motion/confidence.rs:17-21 in f32, left to right."""
    f = np.float32
    return float(f(f(f(blksize * blksize) * f(2.0)) * f(sigma)) / np.sqrt(f(np.pi)))


def thsad(blksize: int, thsad_scale: float) -> float:
    """motion/confidence.rs:27-30 in f32."""
    f = np.float32
    return float(f(f(thsad_scale) * f(blksize * blksize)) * f(0.02))


# ---- camera model (global_oracle.cpp; motion/global/) ---------------------------------------------

MODEL_WORDS = 5
AFFINE_WORDS = 6
NO_PAIR = 0xFFFFFFFF
HIGH_PASS_RADIUS = 8          # global/producer.rs:44-49
ACQUISITION_COARSE_RADIUS = 12  # producer.rs:54-55
ACQUISITION_COARSE_FACTOR = 2   # producer.rs:57-60
MAX_PYRAMID_LEVELS = 3          # motion/search.rs:183


def _i32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def compose_models(models: np.ndarray, gaps: np.ndarray, neighbours: int, max_steps: int,
                   past_neighbours: int) -> np.ndarray:
    """motion/kernels/global.rs:18-119: one prediction (m00, m01, m10, m11, tx, ty) per neighbour
    from the model ring `models` and the gap table `gaps` (ring slots, NO_PAIR for none)."""
    m = np.ascontiguousarray(models, np.float32).reshape(-1)
    g = np.ascontiguousarray(gaps, np.uint32).reshape(-1)
    out = np.zeros(neighbours * AFFINE_WORDS, np.float32)
    l = lib()
    l.orc_compose_models.argtypes = [_fp, _u32p, _fp, C.c_uint32, C.c_uint32, C.c_uint32]
    l.orc_compose_models(_f(m), g.ctypes.data_as(_u32p), _f(out), neighbours, max_steps, past_neighbours)
    return out


def compose_gaps(window_frames, centre: int, max_steps: int, slot_of) -> np.ndarray:
    """global/compose.rs:18-64: the gap table of a window of stream frames, each gap the ring slot
    (`slot_of(newer_frame)`) of a pair that steps exactly one frame, else NO_PAIR."""
    def gap(older):
        return slot_of(window_frames[older + 1]) if window_frames[older + 1] == window_frames[older] + 1 else NO_PAIR

    positions = [p for p in range(len(window_frames)) if p != centre]
    gaps = np.full(len(positions) * max_steps, NO_PAIR, np.uint32)
    for row, p in enumerate(positions):
        dist = abs(p - centre)
        assert dist <= max_steps
        for step in range(dist):
            older = centre - step - 1 if p < centre else centre + step
            gaps[row * max_steps + step] = gap(older)
    return gaps


def block_means(plane: np.ndarray, width: int, height: int, blksize: int, step: int) -> np.ndarray:
    """motion/kernels/global.rs:121-155: each block's mean sample."""
    bx, by = max(-(-width // step), 1), max(-(-height // step), 1)
    src = np.ascontiguousarray(plane, np.float32).reshape(-1)
    out = np.zeros(bx * by, np.float32)
    l = lib()
    l.orc_block_means.argtypes = [_fp, _fp] + [C.c_int] * 6
    l.orc_block_means(_f(src), _f(out), width, height, blksize, step, bx, by)
    return out


def high_pass(plane: np.ndarray, width: int, height: int, radius: int = HIGH_PASS_RADIUS) -> np.ndarray:
    """motion/kernels/pyramid.rs:66-132: the plane minus its (2r+1)^2 box mean, rows then columns."""
    src = np.ascontiguousarray(plane, np.float32).reshape(-1)
    rows = np.zeros_like(src)
    out = np.zeros_like(src)
    l = lib()
    l.orc_high_pass.argtypes = [_fp, _fp, _fp, C.c_int, C.c_int, C.c_int]
    l.orc_high_pass(_f(src), _f(rows), _f(out), width, height, radius)
    return out


def model_fit(field: np.ndarray, width: int, height: int, blksize: int, overlap: int, *, sad: np.ndarray | None = None,
              has_contrast: bool = False, older_to_newer: bool = True, models: np.ndarray | None = None,
              slot: int = 0, prior: int | None = None):
    """global/fit.rs:196-250 (`run_model_fit`): fits one direction of a pair field into ring slot
    `slot` of `models` (updated in place; a one-slot ring when None). `sad` holds the winning SADs,
    then, with `has_contrast`, the window means and the block means, one block count apart. Returns
    (models, state)."""
    step = blksize - overlap
    bx, by = max(-(-width // step), 1), max(-(-height // step), 1)
    f = np.ascontiguousarray(field, np.int32).reshape(-1)
    ring = np.zeros(MODEL_WORDS, np.float32) if models is None else models
    assert ring.dtype == np.float32 and ring.flags["C_CONTIGUOUS"]
    sd = np.ascontiguousarray(sad, np.float32).reshape(-1) if sad is not None else None
    state = np.zeros(8, np.float32)
    l = lib()
    l.orc_model_fit.argtypes = [C.POINTER(C.c_int32), _fp, C.c_int, C.c_uint32, C.c_int] + [C.c_int] * 7 + \
        [_fp, C.c_uint32, _fp]
    l.orc_model_fit(_i32(f), _f(sd) if sd is not None else None, int(has_contrast), bx * by, int(older_to_newer),
                    width, height, blksize, step, bx, by, -1 if prior is None else prior, _f(ring), slot, _f(state))
    return ring, state


def fit_bands(field: np.ndarray, width: int, height: int, blksize: int, overlap: int, *, sad=None,
              has_contrast: bool = False) -> np.ndarray:
    """global.rs:286-392: the four bar bounds (top end, bottom start, left end, right start)."""
    step = blksize - overlap
    bx, by = max(-(-width // step), 1), max(-(-height // step), 1)
    f = np.ascontiguousarray(field, np.int32).reshape(-1)
    sd = np.ascontiguousarray(sad, np.float32).reshape(-1) if sad is not None else None
    bands = np.zeros(4, np.uint32)
    l = lib()
    l.orc_fit_bands.argtypes = [C.POINTER(C.c_int32), _fp, C.c_int, C.c_uint32] + [C.c_int] * 6 + [_u32p]
    l.orc_fit_bands(_i32(f), _f(sd) if sd is not None else None, int(has_contrast), bx * by, width, height, blksize,
                    step, bx, by, bands.ctypes.data_as(_u32p))
    return bands


def pair_models_for(luma_frames, width: int, height: int, **mode) -> "PairModels":
    """A `PairModels` fed every normalised luma frame of a stream in push order (frame i at index i):
    the models are causal, and the engine's ring keeps every model a window reads."""
    pm = PairModels(width, height, **mode)
    for i, f in enumerate(luma_frames):
        pm.push(np.ascontiguousarray(f, np.float32), i)
    return pm


class PairModels:
    """global/producer.rs (`PairModelProducer`): one camera model per adjacent pair of pushed luma
    frames, kept by stream frame (the engine's ring of `held + window + 2` slots never drops a model a
    window still reads). Each push normalised luma loses its local mean, its block means are
    measured, and it is matched against the frame before it: first a deep search (3 levels, coarse
    radius 12 with blocks twice as wide, the search's escalation, the truemotion stage whose SADs
    replace the search's) fitted from scratch, then the mode's own search around that model's
    prediction, fitted again with the first fit as its prior. The first frame of a run, and a frame
    that does not follow the last one pushed, writes identity."""

    def __init__(self, width: int, height: int, *, blksize=16, overlap=8, search_radius=4, levels=2, ceiling=0):
        self.w, self.h = width, height
        self.blksize, self.overlap, self.radius, self.levels = blksize, overlap, search_radius, levels
        self.ceiling = ceiling if ceiling > search_radius else 0
        step = blksize - overlap
        self.bx, self.by = max(-(-width // step), 1), max(-(-height // step), 1)
        lp = lib()
        lp.orc_motion_pyramid_floats.argtypes = [C.c_int] * 4
        lp.orc_motion_pyramid_floats.restype = C.c_int64
        self.pyramid = np.zeros(lp.orc_motion_pyramid_floats(width, height, 2, MAX_PYRAMID_LEVELS), np.float32)
        self.models: dict[int, np.ndarray] = {}
        self.run = None  # (first, last)
        self.means = np.zeros(self.bx * self.by, np.float32)

    def reset(self):
        self.run = None

    def model(self, frame: int) -> np.ndarray:
        return self.models.get(frame, np.array([1, 0, 0, 0, 0], np.float32))

    def _build(self, luma: np.ndarray, slot: int):
        w, h = self.w, self.h
        self.means = block_means(luma, w, h, self.blksize, self.blksize - self.overlap)
        hp = high_pass(luma, w, h)
        lp = lib()
        lp.orc_motion_pyramid_build.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _fp, C.c_int]
        lp.orc_motion_pyramid_build(_f(hp), 1, w, h, 2, 0, MAX_PYRAMID_LEVELS, _f(self.pyramid), slot)

    def push(self, luma: np.ndarray, frame: int):
        """Fits the pair from stream frame `frame - 1` to `frame`; `luma` is the normalised plane."""
        newer = frame % 2
        self._build(np.ascontiguousarray(luma, np.float32).reshape(-1), newer)
        run = self.run
        if run is None or not (run[0] < frame and (run[1] == frame or run[1] + 1 == frame)):
            self.run = (frame, frame)
            self.models[frame] = np.array([1, 0, 0, 0, 0], np.float32)
            return
        self.run = (run[0], frame)
        older = (frame - 1) % 2
        blocks = self.bx * self.by
        th = thsad(self.blksize, 1.0)
        kw = dict(blksize=self.blksize, overlap=self.overlap, search_radius=self.radius, thsad=th, sad_floor=0.0,
                  ceiling=self.ceiling, esc_reads_floor=False)
        ring = np.zeros(MODEL_WORDS, np.float32)
        # producer.rs:435-480: the deep search, ending with the truemotion stage.
        sad = np.zeros(3 * blocks, np.float32)
        sad[2 * blocks:] = self.means
        mv, _ = motion_search(self.pyramid, self.w, self.h, 2, older, [newer], levels=MAX_PYRAMID_LEVELS,
                              field_lambda=1.0, reads_floor=False, sad_out=sad[:2 * blocks],
                              coarse_radius=ACQUISITION_COARSE_RADIUS, coarse_block_factor=ACQUISITION_COARSE_FACTOR,
                              **kw)
        model_fit(mv[0], self.w, self.h, self.blksize, self.overlap, sad=sad, has_contrast=True, models=ring)
        # producer.rs:415-420: the one-step prediction, then the mode's search around it.
        pred = compose_models(ring, np.zeros(1, np.uint32), 1, 1, 0)
        sad2 = np.zeros(3 * blocks, np.float32)
        sad2[2 * blocks:] = self.means
        mv2, _ = motion_search(self.pyramid, self.w, self.h, 2, older, [newer], levels=self.levels, predictions=pred,
                               sad_out=sad2[:2 * blocks], **kw)
        model_fit(mv2[0], self.w, self.h, self.blksize, self.overlap, sad=sad2, has_contrast=True, models=ring,
                  prior=0)
        self.models[frame] = ring.copy()

    def compose_window(self, window_frames, centre: int) -> np.ndarray:
        """nlmeans/denoiser/seeds.rs:136-160: every neighbour's prediction for a window of stream
        frames (positions before `centre` are past neighbours), 2d steps each."""
        nb = len(window_frames) - 1
        frames = sorted(set(window_frames))
        index = {f: i for i, f in enumerate(frames)}
        ring = np.concatenate([self.model(f) for f in frames]).astype(np.float32)
        gaps = compose_gaps(window_frames, centre, nb, lambda f: index[f])
        return compose_models(ring, gaps, nb, nb, centre)

    def compose_pair(self, older: int, newer: int) -> tuple[np.ndarray, np.ndarray]:
        """seeds.rs:104-134: (older-to-newer, newer-to-older) predictions of one pair; a pair that does
        not step exactly one frame predicts no motion."""
        ring = self.model(newer).astype(np.float32)
        gap = np.array([0 if newer == older + 1 else NO_PAIR], np.uint32)
        return compose_models(ring, gap, 1, 1, 0), compose_models(ring, gap, 1, 1, 1)


# ---- NL4D engine over a stream (nl4d/engine.rs, nl4d/denoiser.rs) --------------------------------

def collab_normalise(accum: np.ndarray, wsum: np.ndarray, channels: int) -> np.ndarray:
    """collab/kernels/aggregate.rs:251-290: accum * 5 / wsum in f32, accum itself where wsum is 0."""
    f = np.float32
    acc = accum.reshape(-1, channels).astype(np.float32)
    w = wsum.astype(np.float32)[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        v = (acc * f(5.0)).astype(np.float32) / np.where(w != 0, w, f(1.0))
    return np.where(w != 0, v, acc).astype(np.float32)


def chain_compose(pairs: dict, centre: int, d: int, head_mod: int, step: int, width: int, height: int, bx: int,
                  by: int) -> np.ndarray:
    """motion/kernels/chain.rs: every neighbour's seed walked through the pair ring from the centre;
    `pairs[slot]` holds (older-to-newer, newer-to-older) fields of (blocks, 2)."""
    slots = 2 * d
    seeds = np.zeros((2 * d, bx * by, 2), np.int32)
    for n in range(2 * d):
        logical = n if n < centre else n + 1
        k = logical - centre
        forward = k > 0
        start = (head_mod + (centre if forward else centre - 1)) % slots
        for b in range(bx * by):
            px, py = (b % bx) * step + step // 2, (b // bx) * step + step // 2
            ax = ay = 0
            for i in range(abs(k)):
                slot = (start + i) % slots if forward else (start + slots - i) % slots
                cx, cy = min(max(px, 0), width - 1), min(max(py, 0), height - 1)
                hb = min(cy // step, by - 1) * bx + min(cx // step, bx - 1)
                hop = pairs[slot][0 if forward else 1][hb]
                ax, ay, px, py = ax + int(hop[0]), ay + int(hop[1]), px + int(hop[0]), py + int(hop[1])
            seeds[n, b] = (ax, ay)
    return seeds


def map_luma_fields(luma_mv: np.ndarray, luma_grid: tuple[int, int, int, int], chroma_grid: tuple[int, int, int, int],
                    shift_x: int, shift_y: int) -> np.ndarray:
    """motion/kernels/chroma_map.rs (`mc_map_luma_fields`): every field of `luma_mv` (n, blocks, 2)
    onto the chroma block grid; grids are (blocks_x, blocks_y, step, blksize). Each chroma block
    takes the per-component lower median of the luma blocks inside the area it covers (clamped to
    the luma grid), divided by the subsampling and rounded half away from zero."""
    lbx, lby, lstep, lblk = luma_grid
    cbx, cby, cstep, cblk = chroma_grid
    covers_x = max((cblk << shift_x) - lblk, 0) // lstep + 1
    covers_y = max((cblk << shift_y) - lblk, 0) // lstep + 1
    n = luma_mv.shape[0]
    lum = luma_mv.reshape(n, lby, lbx, 2)
    out = np.zeros((n, cby * cbx, 2), np.int32)

    def scale_down(v, shift):
        if shift == 0:
            return v
        r = (abs(v) + (1 << (shift - 1))) // (1 << shift)
        return -r if v < 0 else r

    for row in range(cby):
        for col in range(cbx):
            ox, oy = (col * cstep) << shift_x, (row * cstep) << shift_y
            sc, sr = ox // lstep, oy // lstep
            lc, lr = min(sc + covers_x - 1, lbx - 1), min(sr + covers_y - 1, lby - 1)
            fc, fr = min(sc, lc), min(sr, lr)
            live = [(fr + i // covers_x, fc + i % covers_x) for i in range(covers_x * covers_y)
                    if fc + i % covers_x <= lc and fr + i // covers_x <= lr]
            for f in range(n):
                vals = np.array([lum[f, r, c] for r, c in live], np.int64)
                mx = int(np.sort(vals[:, 0])[(len(vals) - 1) // 2])
                my = int(np.sort(vals[:, 1])[(len(vals) - 1) // 2])
                out[f, row * cbx + col] = (scale_down(mx, shift_x), scale_down(my, shift_y))
    return out


class MotionShare:
    """The luma pass's window fields shared with the chroma pass of one engine (motion/luma_ring.rs):
    a luma stream writes each window's field, keyed by engine call and by the centre's stream frame
    modulo the ring size (a later window of the same call overwrites the slot); a chroma stream of
    the same calls reads the slot of its window's centre frame, mapped onto its own block grid."""

    def __init__(self, luma_grid, chroma_grid, shift_x, shift_y):
        self.luma_grid, self.chroma_grid = luma_grid, chroma_grid
        self.shift_x, self.shift_y = shift_x, shift_y
        self.calls: dict[int, dict[int, tuple[int, np.ndarray]]] = {}

    def write(self, call: int, slot: int, frame: int, mv: np.ndarray):
        self.calls.setdefault(call, {})[slot] = (frame, mv.copy())

    def read(self, call: int, slot: int, frame: int) -> np.ndarray:
        held = self.calls.get(call, {}).get(slot)
        assert held is not None and held[0] == frame, "the luma pass has not shared this frame's motion"
        return map_luma_fields(held[1], self.luma_grid, self.chroma_grid, self.shift_x, self.shift_y)


def nl4d_stream(frames: list[np.ndarray], d: int, sigma: float, *, blksize=16, overlap=8, search_radius=4,
                levels=2, refine=2, spatial_radius=9, lambda_ht=4.158, c_min=0.05, kaiser_beta=2.0,
                pool_ratio: float | None = None, thsad_scale=1.0, context: int = 0, chained: bool = False,
                refine_radius: int = 2, noise=None, field_lambda: float = 1.0, share_writes: MotionShare | None = None,
                share_reads: MotionShare | None = None, ceiling: int = 0, camera_model: bool = True,
                models: "PairModels | None" = None, wiener: bool = False) -> list[np.ndarray]:
    """The NL4D engine with a pinned sigma and Direct or Chained motion over a
    stream of (H, W, C) f32 frames; returns the emitted (H, W, C) f32 frames in order. With
    `field_lambda` > 0 the truemotion stage ends the Direct window search (reading the window's SAD
    floor) and each pair search (without it); the chained refine runs none
    (nlmeans/dispatch/motion.rs:201-206, denoiser/stages.rs:146-197).

    It follows nl4d/engine.rs:287-381 and nl4d/denoiser.rs:370-596: a shifted-edge ring of 2d+1
    slots; when the ring first fills at a scene start, head passes centred on logical 0..d-1, then
    one pass centred on the middle slot per push; after more than d passes each middle pass
    completes the region d slots behind it; at the end, tail passes centred on d+1..2d (or, for a
    stream shorter than the ring, on every real frame after padding with the last frame). The
    first `context` frames are priming pushes (no head passes). With `noise`, a function of a pass's
    centre stream frame returning (sigma or per-channel sigmas, weight_scale, sad_floor), optionally
    followed by curve and
    colour, each pass reads those (the automatic estimate's fold around that frame) instead of the
    pinned sigma's; `curve` is the 16 luma noise-curve ratios, or None while the fold's curve flag
    is clear, and `colour` the (gain tables, centre block means, 8-bit scale) of collab_fused. With `share_writes`
    each window's field is shared for a chroma stream; with `share_reads` the window's motion is the
    shared luma field of the centre frame, searched one pixel around at one level with confidence
    (nlmeans/dispatch/motion.rs:231-310), and no motion of this plane's own is searched. With
    `camera_model` a pass that searches its own motion also searches around the camera models
    fitted on channel 0 of the pushed frames (`models`, else a `PairModels` fed every frame in
    order), as in `nlm_stream_mc`. `wiener` adds the empirical Wiener stage to every pass."""
    h, w, c = frames[0].shape
    tf = 2 * d + 1
    step = blksize - overlap
    bx, by = max(-(-w // step), 1), max(-(-h // step), 1)
    ring = np.zeros((tf, h, w, c), np.float32)
    accum = np.zeros((tf, h * w * c), np.int64)
    wsum = np.zeros((tf, h * w), np.int64)
    st = dict(head=0, loaded=0, real=0, passes=0, cont=context > 0, call=0)
    if share_reads is not None:
        chained, levels = False, 1
    if camera_model and share_reads is None and models is None and d > 0:
        models = pair_models_for([f[..., 0] for f in frames], w, h, blksize=blksize, overlap=overlap,
                                 search_radius=search_radius, levels=levels, ceiling=ceiling)
    if not camera_model or share_reads is not None:
        models = None
    slot_frames = [0] * tf
    zeroed = [False] * tf
    sad_floor = sad_noise_floor(blksize, sigma)
    th = thsad(blksize, thsad_scale)

    def phys(logical):
        return (st["head"] % tf + logical) % tf

    def run_pass(centre, clear):
        cs = phys(centre)
        if clear == "whole":
            for s in range(tf):
                accum[s] = 0
                wsum[s] = 0
        elif clear == "newest":
            newest = (cs + d) % tf
            if not zeroed[newest]:
                accum[newest] = 0
                wsum[newest] = 0
        for i in range(tf):
            zeroed[i] = False
        st["passes"] += 1
        slots = [phys(l) for l in range(tf) if l != centre]
        p_sigma, p_weight, p_floor, p_curve, p_colour = sigma, None, sad_floor, None, None
        if noise is not None:
            p_sigma, p_weight, p_floor, *rest = noise(slot_frames[cs])
            p_curve = rest[0] if rest else None
            p_colour = rest[1] if len(rest) > 1 else None
        pyr = motion_pyramid(ring.reshape(-1), c, w, h, levels)
        if share_reads is not None:
            mapped = share_reads.read(st["call"], slot_frames[cs] % tf, slot_frames[cs])
            mv, conf = motion_search(pyr, w, h, tf, cs, slots, blksize=blksize, overlap=overlap,
                                     search_radius=1, levels=1, confidence=True, sad_floor=p_floor, thsad=th,
                                     seeds=mapped)
        elif chained:
            seeds = chain_compose(pairs, centre, d, st["head"] % (2 * d), step, w, h, bx, by)
            mv, conf = motion_search(pyr, w, h, tf, cs, slots, blksize=blksize, overlap=overlap,
                                     search_radius=refine_radius, levels=levels, confidence=True,
                                     sad_floor=p_floor, thsad=th, seeds=seeds, ceiling=ceiling, esc_reads_floor=True)
        else:
            pred = models.compose_window([slot_frames[phys(l)] for l in range(tf)], centre) if models is not None else None
            mv, conf = motion_search(pyr, w, h, tf, cs, slots, blksize=blksize, overlap=overlap,
                                     search_radius=search_radius, levels=levels, confidence=True,
                                     sad_floor=p_floor, thsad=th, field_lambda=field_lambda, reads_floor=True,
                                     ceiling=ceiling, esc_reads_floor=True, predictions=pred)
        if share_writes is not None:
            share_writes.write(st["call"], slot_frames[cs] % tf, slot_frames[cs], mv)
        acc, ws, _ = collab_fused(ring.reshape(-1), w, h, c, centre_slot=cs, radius=d, mv_field=mv.reshape(-1),
                                  confidence=conf.reshape(-1), neighbour_slots=np.array(slots, np.uint32),
                                  c_min=c_min, refine=refine, spatial_radius=spatial_radius, k_max=8,
                                  sigma=tuple(p_sigma) if isinstance(p_sigma, (tuple, list)) else (p_sigma,) * c,
                                  weight_scale_override=p_weight, lambda_ht=lambda_ht,
                                  kaiser_beta=kaiser_beta, noise_curve=p_curve, colour=p_colour,
                                  pooled=pool_ratio, blksize=blksize, blk_step=step, blocks_x=bx, blocks_y=by,
                                  mv_stride=bx * by * 2, conf_stride=bx * by, wiener=wiener)
        accum[:] += acc.reshape(tf, -1)
        wsum[:] += ws.reshape(tf, -1)

    def read_region(slot):
        out = collab_normalise(accum[slot].astype(np.int32), wsum[slot].astype(np.int32), c).reshape(h, w, c)
        accum[slot] = 0
        wsum[slot] = 0
        zeroed[slot] = True
        return out

    pairs = {i: (np.zeros((bx * by, 2), np.int32), np.zeros((bx * by, 2), np.int32)) for i in range(2 * d)}

    def pair_analyse(newer):
        # nlmeans/denoiser/stages.rs:146-197: both directions into pair slot head mod 2d.
        if not chained or st["head"] == 0:
            return
        older = (newer + tf - 1) % tf
        pyr = motion_pyramid(ring.reshape(-1), c, w, h, levels)
        kw = dict(blksize=blksize, overlap=overlap, search_radius=search_radius, levels=levels, thsad=th,
                  field_lambda=field_lambda, reads_floor=False, ceiling=ceiling)
        o2n, n2o = models.compose_pair(slot_frames[older], st["real"]) if models is not None else (None, None)
        fwd, _ = motion_search(pyr, w, h, tf, older, [newer], predictions=o2n, **kw)
        bwd, _ = motion_search(pyr, w, h, tf, newer, [older], predictions=n2o, **kw)
        pairs[st["head"] % (2 * d)] = (fwd[0], bwd[0])

    def push(frame):
        s = st["head"] % tf
        ring[s] = frame
        pair_analyse(s)
        slot_frames[s] = st["real"]
        st["head"] += 1
        st["loaded"] = min(st["loaded"] + 1, tf)
        st["real"] += 1

    outs = []
    for i, frame in enumerate(frames):
        st["call"] = i
        push(frame)
        if i < context or st["loaded"] < tf:
            continue
        clear = "whole" if st["passes"] == 0 else "newest"
        if st["passes"] == 0 and not st["cont"]:
            for centre in range(d):
                run_pass(centre, clear)
                clear = "none"
        run_pass(d, clear)
        if st["passes"] > d:
            outs.append(read_region((phys(d) + tf - d) % tf))
    st["call"] = len(frames)
    emit = min(st["real"], 2 * d)
    if emit == 0:
        return outs
    short = st["real"] < tf
    if short:
        while st["loaded"] < tf:
            last, nxt = (st["head"] - 1) % tf, st["head"] % tf
            ring[nxt] = ring[last]
            if chained:
                pairs[st["head"] % (2 * d)] = (np.zeros((bx * by, 2), np.int32), np.zeros((bx * by, 2), np.int32))
            slot_frames[nxt] = slot_frames[last]
            st["head"] += 1
            st["loaded"] += 1
    centres = range(emit) if short else range(d + 1, 2 * d + 1)
    last_real = emit - 1 if short else 2 * d
    clear = "whole" if (short or st["passes"] == 0) else "none"
    for centre in centres:
        run_pass(centre, clear)
        clear = "none"
    for logical in range(last_real + 1 - emit, last_real + 1):
        outs.append(read_region(phys(logical)))
    return outs


# ---- Immerkær spatial noise estimate (noise_oracle.cpp) ------------------------------------------

def immerkaer_scale() -> float:
    """noise/spatial.rs:142-144: sqrt(pi / 2) in f32."""
    return float(np.sqrt(np.float32(np.pi / 2)))


def immerkaer(frame: np.ndarray, channels: int, width: int, height: int):
    """Returns (partials, totals[2], sigma_low[2]) of one (H, W, C) f32 frame."""
    l = lib()
    l.orc_immerkaer_partials_len.argtypes = [C.c_int, C.c_int]
    l.orc_immerkaer_partials_len.restype = C.c_int64
    l.orc_immerkaer_partials.argtypes = [_fp, C.c_int, C.c_int, C.c_int, _fp]
    l.orc_immerkaer_totals.argtypes = [_fp, C.c_int, _fp]
    l.orc_immerkaer_sigma_low.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_float, _fp]
    fr = np.ascontiguousarray(frame, np.float32)
    partials = np.zeros(l.orc_immerkaer_partials_len(width, height), np.float32)
    l.orc_immerkaer_partials(_f(fr), channels, width, height, _f(partials))
    totals = np.zeros(2, np.float32)
    l.orc_immerkaer_totals(_f(partials), partials.size // 2, _f(totals))
    low = np.zeros(2, np.float32)
    l.orc_immerkaer_sigma_low(_f(partials), channels, width, height, immerkaer_scale(), _f(low))
    return partials, totals, low


def immerkaer_sigma_low_from_partials(partials: np.ndarray, channels: int, width: int, height: int) -> np.ndarray:
    l = lib()
    l.orc_immerkaer_sigma_low.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_float, _fp]
    low = np.zeros(2, np.float32)
    l.orc_immerkaer_sigma_low(_f(np.ascontiguousarray(partials, np.float32)), channels, width, height,
                              immerkaer_scale(), _f(low))
    return low


# ---- automatic noise estimate (noise_estimate_oracle.cpp) ------------------------------------------

READING_WORDS = 30
STATE_WORDS = 32
DERIVED_WORDS = 11
NOISE_WINDOW_RADIUS = 8
LOOKAHEAD_FRAMES = 8
RECIPROCAL_FLOOR = 1e-12


def _noise_lib():
    l = lib()
    l.orc_noise_record_len.argtypes = [C.c_int]
    l.orc_noise_record_len.restype = C.c_int
    l.orc_min_static_blocks.argtypes = [C.c_uint32]
    l.orc_min_static_blocks.restype = C.c_uint32
    l.orc_temporal_stats.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_int, C.c_int, _fp]
    l.orc_noise_reading.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _fp]
    l.orc_temporal_stats_mc.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_int,
                                        C.c_int, C.c_int, _fp]
    l.orc_fold_words.argtypes = [C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float, C.c_int, C.c_float,
                                 C.c_float, C.c_float, C.c_float, C.c_int, C.c_float, C.c_float, C.c_float, _fp]
    l.orc_noise_fold.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_int, _fp, C.c_int, C.c_int, _fp, _fp, _fp, _fp]
    l.orc_correlation_factor.argtypes = [C.c_float, _fp]
    l.orc_correlation_factor.restype = C.c_float
    return l


def noise_record_len(channels: int) -> int:
    return _noise_lib().orc_noise_record_len(channels)


def stats_blocks(width: int, height: int) -> tuple[int, int]:
    return -(-width // 16), -(-height // 16)


def min_static_blocks(total: int) -> int:
    return int(_noise_lib().orc_min_static_blocks(total))


def temporal_stats(new: np.ndarray, prev: np.ndarray, channels: int, width: int, height: int,
                   luma_fields: bool = False) -> np.ndarray:
    """The temporal residual records of `new` against `prev`, (H, W, C) f32 frames; with
    `luma_fields`, each block's four 8x8 quarter records as well."""
    bx, by = stats_blocks(width, height)
    out = np.zeros(bx * by * noise_record_len(channels), np.float32)
    _noise_lib().orc_temporal_stats(_f(np.ascontiguousarray(new, np.float32)),
                                    _f(np.ascontiguousarray(prev, np.float32)), channels, width, height,
                                    int(luma_fields), _f(out))
    return out


def temporal_stats_mc(new: np.ndarray, prev: np.ndarray, channels: int, width: int, height: int, mv: np.ndarray,
                      mv_blocks: tuple[int, int], step: int, luma_fields: bool = False) -> np.ndarray:
    """The records of `new` against `prev` along the motion field `mv` ((bx * by, 2) int32)."""
    bx, by = stats_blocks(width, height)
    out = np.zeros(bx * by * noise_record_len(channels), np.float32)
    field = np.ascontiguousarray(mv, np.int32).reshape(-1)
    _noise_lib().orc_temporal_stats_mc(_f(np.ascontiguousarray(new, np.float32)),
                                       _f(np.ascontiguousarray(prev, np.float32)), channels, width, height,
                                       field.ctypes.data_as(C.POINTER(C.c_int32)), mv_blocks[0], mv_blocks[1], step,
                                       int(luma_fields), _f(out))
    return out


def noise_reading(records: np.ndarray | None, imm_low, channels: int, width: int, height: int,
                  temporal: bool, curve: bool = False) -> np.ndarray:
    """One slot's READING_WORDS reading from its records (None without temporal stats) and its two
    Immerkaer lower quartiles; with `curve` (records carrying the luma fields), the noise curve."""
    out = np.zeros(READING_WORDS, np.float32)
    low = np.ascontiguousarray(np.asarray(imm_low, np.float32).reshape(2))
    rec = _f(np.ascontiguousarray(records, np.float32)) if records is not None else None
    _noise_lib().orc_noise_reading(rec, _f(low), channels, width, height, int(temporal), int(curve), _f(out))
    return out


def fold_words(width: int, height: int, *, sigma_scale=1.0, curve_applies=False, g_max=0.0,
               weight_floor=RECIPROCAL_FLOOR, h2_per_inverse_variance=None, h2_fixed=0.0, pilot_h2_factor=1.0,
               offset_per_variance=0.0, main_offset=True, sad_per_sigma=0.0,
               confidence_sad_per_sigma=0.0) -> np.ndarray:
    """noise/fold.rs:118-146: the 16 fold settings words."""
    out = np.zeros(16, np.float32)
    _noise_lib().orc_fold_words(width, height, sigma_scale, int(curve_applies), g_max, weight_floor,
                                int(h2_per_inverse_variance is not None), h2_per_inverse_variance or 0.0, h2_fixed,
                                pilot_h2_factor, offset_per_variance, int(main_offset), sad_per_sigma,
                                confidence_sad_per_sigma, immerkaer_scale(), _f(out))
    return out


def correlation_factor(rho: float, settings: np.ndarray) -> float:
    return float(_noise_lib().orc_correlation_factor(rho, _f(np.ascontiguousarray(settings, np.float32))))


def noise_fold(records: np.ndarray, results: np.ndarray, capacity: int, first: int, last: int,
               settings: np.ndarray, channels: int, table_radius: int = 0):
    """One window fold over history frames first..=last (frame f in slot f % capacity). Returns
    (state, derived, spatial_table, pilot_table)."""
    side = 2 * table_radius + 1
    state = np.zeros(STATE_WORDS, np.float32)
    derived = np.zeros(DERIVED_WORDS, np.float32)
    spatial = np.zeros(side * side, np.float32)
    pilot = np.zeros(side * side, np.float32)
    _noise_lib().orc_noise_fold(_f(np.ascontiguousarray(records, np.float32)),
                                _f(np.ascontiguousarray(results, np.float32)), capacity, first, last,
                                _f(np.ascontiguousarray(settings, np.float32)), channels, table_radius, _f(state),
                                _f(derived), _f(spatial), _f(pilot))
    return state, derived, spatial, pilot


def noise_readings(frames: list[np.ndarray], channels: int, width: int, height: int, temporal: bool,
                   luma_fields: bool = False):
    """Every frame's reading and Immerkaer totals, each read against the frame before it (the first
    frame's records are zero), as the look-ahead reads them without motion compensation
    (nlmeans/denoiser/lookahead.rs:425-444)."""
    readings, totals = [], []
    for i, f in enumerate(frames):
        _, tot, low = immerkaer(f, channels, width, height)
        rec = None
        if temporal:
            if i == 0:
                rec = np.zeros(stats_blocks(width, height)[0] * stats_blocks(width, height)[1]
                               * noise_record_len(channels), np.float32)
            else:
                rec = temporal_stats(f, frames[i - 1], channels, width, height, luma_fields)
        readings.append(noise_reading(rec, low, channels, width, height, temporal, luma_fields))
        totals.append(tot)
    return readings, totals


def noise_readings_mc(frames: list[np.ndarray], channels: int, width: int, height: int, *, blksize: int,
                      overlap: int, search_radius: int, levels: int, thsad: float = 0.0, ceiling: int = 0,
                      luma_fields: bool = False, records_out: list | None = None, camera_model: bool = True,
                      models: "PairModels | None" = None):
    """Every frame's reading as a motion-compensated look-ahead takes it
    (nlmeans/denoiser/lookahead.rs:283-319, 425-458, 543-605): frame i >= 1 is searched against
    frame i - 1 (newer to older) and read along that field; frame 1 is also searched older to newer
    and frame 0 re-read along it. Frame 0 keeps its Immerkaer words from its own read. Returns
    (readings, Immerkaer totals). With `records_out`, each frame's final temporal records are
    appended to it. With `camera_model` each pair search also searches around the pair's camera-model
    prediction (lookahead.rs:310-316), the models fitted on channel 0 of the frames."""
    step = blksize - overlap
    mb = (max(-(-width // step), 1), max(-(-height // step), 1))
    # With `ceiling` the pair searches escalate, measuring their own floor (lookahead.rs:509-515).
    kw = dict(blksize=blksize, overlap=overlap, search_radius=search_radius, levels=levels, thsad=thsad,
              ceiling=ceiling)
    rec_len = stats_blocks(width, height)[0] * stats_blocks(width, height)[1] * noise_record_len(channels)
    if camera_model and models is None:
        models = pair_models_for([np.asarray(f, np.float32).reshape(height, width, channels)[..., 0] for f in frames],
                                 width, height, blksize=blksize, overlap=overlap, search_radius=search_radius,
                                 levels=levels, ceiling=ceiling)
    if not camera_model:
        models = None
    readings, totals, lows = [], [], []
    for i, f in enumerate(frames):
        _, tot, low = immerkaer(f, channels, width, height)
        totals.append(tot)
        lows.append(low)
        if i == 0:
            readings.append(noise_reading(np.zeros(rec_len, np.float32), low, channels, width, height, True,
                                          luma_fields))
            if records_out is not None:
                records_out.append(np.zeros(rec_len, np.float32))
            continue
        pair = np.stack([np.ascontiguousarray(frames[i - 1], np.float32),
                         np.ascontiguousarray(f, np.float32)]).reshape(-1)
        pyr = motion_pyramid(pair, channels, width, height, levels)
        o2n, n2o = models.compose_pair(i - 1, i) if models is not None else (None, None)
        newer_to_older, _ = motion_search(pyr, width, height, 2, 1, [0], predictions=n2o, **kw)
        rec = temporal_stats_mc(f, frames[i - 1], channels, width, height, newer_to_older[0], mb, step, luma_fields)
        readings.append(noise_reading(rec, low, channels, width, height, True, luma_fields))
        if records_out is not None:
            records_out.append(rec)
        if i == 1:
            older_to_newer, _ = motion_search(pyr, width, height, 2, 0, [1], predictions=o2n, **kw)
            rec0 = temporal_stats_mc(frames[0], f, channels, width, height, older_to_newer[0], mb, step, luma_fields)
            readings[0] = noise_reading(rec0, lows[0], channels, width, height, True, luma_fields)
            if records_out is not None:
                records_out[0] = rec0
    return readings, totals


def noise_window(centre: int, newest: int) -> tuple[int, int]:
    """noise/history.rs:31-44 (`WindowBounds::around`)."""
    return max(centre - NOISE_WINDOW_RADIUS, 0), min(centre + NOISE_WINDOW_RADIUS, newest)


def fold_stream(readings, totals, settings, channels: int, table_radius: int, temporal_radius: int):
    """The fold of every centre frame of a stream of n frames: window around(c, n - 1) over a
    history of 17 + d slots, as the NLMeans front folds before each pass. Returns a list of
    (state, derived, spatial_table, pilot_table)."""
    n = len(readings)
    cap = 2 * NOISE_WINDOW_RADIUS + 1 + temporal_radius
    out = []
    for c in range(n):
        first, last = noise_window(c, n - 1)
        records = np.zeros(cap * READING_WORDS, np.float32)
        results = np.zeros(cap * 2, np.float32)
        for f in range(first, last + 1):
            records[(f % cap) * READING_WORDS:(f % cap + 1) * READING_WORDS] = readings[f]
            results[(f % cap) * 2:(f % cap) * 2 + 2] = totals[f]
        out.append(noise_fold(records, results, cap, first, last, settings, channels, table_radius))
    return out


def nlm_stream_hq_auto(frames: list[np.ndarray], d: int, a: int, s: int, strength: float, *, wref: float = 1.0,
                       auto_strength: bool = True, noise_floor: bool = True, temporal_confidence: bool = True,
                       thsad_scale: float = 1.0, sigma_scale: float = 1.0, fp64: bool = False):
    """NLMeans-HQ with the automatic noise estimate over a stream with repeat edges: every frame is
    read against the one before it (nlmeans/denoiser/lookahead.rs:425-444), each output frame's
    window of readings is folded around its centre (nlmeans/denoiser/noise.rs:171-185) into h2, the
    offset table at the folded correlation and the confidence SAD floor (noise/fold.rs, derived.rs),
    and the frame is denoised with them. Returns (outputs, folds)."""
    h, w, c = frames[0].shape
    f = np.float32
    area = f((2 * s + 1) ** 2)
    readings, totals = noise_readings(frames, c, w, h, d >= 1)
    # nlmeans/denoiser/noise.rs:200-246: each coefficient at a sigma of 1.
    h2_unit = h2_inv_norm(float(f(strength) * f(1.0) * f(255.0)), s)
    scale = f(3.0) if c == 1 else f(1.5)
    offset_unit = float(((f(2.0) * scale) * f(1.0)) * area) if noise_floor else 0.0
    conf = temporal_confidence and d > 0
    settings = fold_words(w, h, sigma_scale=sigma_scale, h2_per_inverse_variance=h2_unit if auto_strength else None,
                          h2_fixed=h2_inv_norm(strength, s), offset_per_variance=offset_unit,
                          confidence_sad_per_sigma=sad_noise_floor(16, 1.0) if conf else 0.0)
    folds = fold_stream(readings, totals, settings, c, a, d)
    n = len(frames)
    outs = []
    for i in range(n):
        window = [frames[min(max(i + k, 0), n - 1)] for k in range(-d, d + 1)]
        derived, lut = folds[i][1], folds[i][2]
        cf, blocks = None, (1, 1)
        if conf:
            cf, blocks = hq_confidence(window, d, 0.0, thsad_scale, sad_floor=float(derived[5]))
        outs.append(nlm_frame(window, d, a, s, float(derived[6]), noise_offset=float(derived[8]), lut=lut, conf=cf,
                              conf_step=8, blocks=blocks, wref=wref, fp64=fp64))
    return outs, folds


def fold_at(readings, totals, settings, channels: int, table_radius: int, temporal_radius: int, centre: int,
            newest: int):
    """The fold of the window around stream frame `centre` when frames 0..=newest are recorded
    (noise/history.rs:31-44 over a history of 17 + d slots). Returns (state, derived, spatial, pilot)."""
    cap = 2 * NOISE_WINDOW_RADIUS + 1 + temporal_radius
    first, last = noise_window(centre, newest)
    records = np.zeros(cap * READING_WORDS, np.float32)
    results = np.zeros(cap * 2, np.float32)
    for f in range(first, last + 1):
        records[(f % cap) * READING_WORDS:(f % cap + 1) * READING_WORDS] = readings[f]
        results[(f % cap) * 2:(f % cap) * 2 + 2] = totals[f]
    return noise_fold(records, results, cap, first, last, settings, channels, table_radius)


LOOKAHEAD_FRAMES = 8


def nlm_stream_hq_auto_pilot(frames: list[np.ndarray], d: int, a: int, s: int, strength: float,
                             strength_scale: float, *, wref: float = 1.0, auto_strength: bool = True,
                             noise_floor: bool = True, temporal_confidence: bool = True, thsad_scale: float = 1.0,
                             sigma_scale: float = 1.0, fp64: bool = False):
    """NLMeans-HQ with the automatic noise estimate and the spatial-NLM pilot, replayed event by
    event as the front runs it, since each pilot reads the derived words of the latest fold:
      - a push first releases the oldest of 8 look-ahead frames into the ring (lookahead.rs:226-259),
        then reads the pushed frame (recorded = pushes so far), then denoises the window centre if
        the ring is full, folding around it first (dispatch/mod.rs:640-644);
      - a frame entering the ring is piloted with the current derived words (stages.rs:29-40); the
        stream's first frame folds the window around frame 0 first (noise.rs:147-165) and its d
        leading-edge copies are piloted with the same words (ring.rs:103-180);
      - the tail releases the held frames, then duplicates the last frame, each re-piloted with the
        words of that moment, one output per step (denoiser/mod.rs:534-573).
    The pilot uses derived word 7 and the fold's pilot table; the main pass word 6, offset word 8
    (0 under the pilot) and the spatial table. Returns (outputs, [(centre, derived) per output])."""
    h, w, c = frames[0].shape
    f = np.float32
    area = f((2 * s + 1) ** 2)
    n = len(frames)
    readings, totals = noise_readings(frames, c, w, h, d >= 1)
    h2_unit = h2_inv_norm(float(f(strength) * f(1.0) * f(255.0)), s)
    scale = f(3.0) if c == 1 else f(1.5)
    offset_unit = float(((f(2.0) * scale) * f(1.0)) * area) if noise_floor else 0.0
    conf = temporal_confidence and d > 0
    sc = f(strength_scale)
    settings = fold_words(w, h, sigma_scale=sigma_scale, h2_per_inverse_variance=h2_unit if auto_strength else None,
                          h2_fixed=h2_inv_norm(strength, s), pilot_h2_factor=float(f(1.0) / (sc * sc)),
                          offset_per_variance=offset_unit, main_offset=False,
                          confidence_sad_per_sigma=sad_noise_floor(16, 1.0) if conf else 0.0)
    state = {"fold": None, "recorded": 0}
    entries = []  # (stream frame, reference) per ring entry, oldest first
    outs, used = [], []

    def pilot(frame_idx):
        derived, pilot_table = state["fold"][1], state["fold"][3]
        return nlm_frame([frames[frame_idx]], 0, a, s, float(derived[7]), lut=pilot_table, wref=wref)

    def enter(frame_idx):
        if not entries:
            state["fold"] = fold_at(readings, totals, settings, c, a, d, 0, state["recorded"] - 1)
        entries.append((frame_idx, pilot(frame_idx)))
        if len(entries) == 1:
            entries.extend([entries[0]] * d)

    def denoise(newest):
        if len(entries) < 2 * d + 1:
            return
        window = entries[-(2 * d + 1):]
        centre = window[d][0]
        fold = fold_at(readings, totals, settings, c, a, d, centre, newest)
        state["fold"] = fold
        derived, lut = fold[1], fold[2]
        inputs = [frames[e[0]] for e in window]
        cf, blocks = None, (1, 1)
        if conf:
            cf, blocks = hq_confidence(inputs, d, 0.0, thsad_scale, sad_floor=float(derived[5]))
        outs.append(nlm_frame(inputs, d, a, s, float(derived[6]), noise_offset=float(derived[8]), lut=lut, conf=cf,
                              conf_step=8, blocks=blocks, wref=wref, fp64=fp64, refs=[e[1] for e in window]))
        used.append((centre, derived))

    for i in range(n):
        if i >= LOOKAHEAD_FRAMES:
            enter(i - LOOKAHEAD_FRAMES)
        state["recorded"] = i + 1
        denoise(i)
    held = list(range(max(n - LOOKAHEAD_FRAMES, 0), n))
    while len(outs) < n:
        before = len(outs)
        while len(outs) == before:
            if held:
                enter(held.pop(0))
            else:
                last = entries[-1][0]
                entries.append((last, pilot(last)))
            denoise(n - 1)
    return outs, used


# ---- NLMeans adjoint (nlm_backward_oracle.cpp) -----------------------------------------------------

def nlm_backward(window: list[np.ndarray], d: int, a: int, s: int, strength: float, grad_out: np.ndarray,
                 wref: float = 1.0, pair_offset: float = 0.0, spatial_offset: float = 0.0):
    """FP64 dL/d(window frames) (2d+1, H, W, C) and dL/d(strength) for dL/d(out) = grad_out."""
    h, w, c = window[0].shape
    frames = [np.ascontiguousarray(f, np.float32) for f in window]
    arr = (_fp * len(frames))(*[_f(f) for f in frames])
    g = np.ascontiguousarray(grad_out, np.float64)
    gf = np.zeros((2 * d + 1, h, w, c), np.float64)
    gs = C.c_double(0.0)
    l = lib()
    l.orc_nlm_backward_f64.argtypes = [_fpp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                       C.c_double, C.c_double, C.c_double, _dp, _dp, C.POINTER(C.c_double)]
    l.orc_nlm_backward_f64(arr, w, h, c, d, a, s, strength, wref, pair_offset, spatial_offset,
                           g.ctypes.data_as(_dp), gf.ctypes.data_as(_dp), C.byref(gs))
    return gf, gs.value


def nlm_forward_f64(window: list[np.ndarray], d: int, a: int, s: int, strength: float, wref: float = 1.0,
                    pair_offset: float = 0.0, spatial_offset: float = 0.0) -> np.ndarray:
    """The FP64 forward with h2 taken in FP64 from `strength` (for finite differences)."""
    h2 = 65025.0 / (3.0 * strength * strength * (2 * s + 1) ** 2)
    side = 2 * a + 1
    lut = np.full(side * side, spatial_offset, np.float32)
    lut[a * side + a] = 0.0
    return nlm_frame(window, d, a, s, h2, noise_offset=pair_offset, lut=lut if spatial_offset else None, wref=wref,
                     fp64=True)


# ---- the colour grain gains (noise/colour.rs, noise/kernels/colour.rs, colour_fit.rs) ----------

COLOUR_CELLS = 976
COLOUR_CELL_WORDS = 69
COLOUR_FIT_PLANE_WORDS = 22
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)


def _colour_lib():
    l = lib()
    l.orc_colour_records.argtypes = [C.c_int, C.c_int]
    l.orc_colour_records.restype = C.c_int
    l.orc_colour_cell.argtypes = [C.c_float, C.c_float, C.c_float]
    l.orc_colour_cell.restype = C.c_uint32
    l.orc_log_mirror.argtypes = [C.c_float]
    l.orc_log_mirror.restype = C.c_float
    l.orc_atan2_mirror.argtypes = [C.c_float, C.c_float]
    l.orc_atan2_mirror.restype = C.c_float
    l.orc_colour_means.argtypes = [_u32p, _u32p, _u32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_float, C.c_float, _fp, _fp]
    l.orc_colour_accumulate.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, _i32p]
    l.orc_colour_window.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, _fp]
    l.orc_colour_levels.argtypes = [_fp, _fp, C.c_int, C.c_int, _fp]
    l.orc_colour_fit.argtypes = [_fp, C.c_int, C.c_int, _fp, C.c_int, _fp, _fp, _fp]
    l.orc_colour_lookup.argtypes = [_fp, _fp, C.c_int, _fp, _fp]
    return l


def colour_records(planes: int, luma: bool) -> int:
    """The cell and extra records of one frame's sums: `planes` x 976 cells, then 16 luma
    calibration records or one chroma record per plane."""
    return _colour_lib().orc_colour_records(planes, int(luma))


def colour_cell(luma: float, cb: float, cr: float) -> int:
    return int(_colour_lib().orc_colour_cell(luma, cb, cr))


def log_mirror(x: float) -> float:
    return float(_colour_lib().orc_log_mirror(x))


def atan2_mirror(y: float, x: float) -> float:
    return float(_colour_lib().orc_atan2_mirror(y, x))


def colour_means(luma: np.ndarray, cb: np.ndarray, cr: np.ndarray, width: int, height: int, shift_x: int,
                 shift_y: int, samples_per_word: int, is_float: bool, eight_bit_scale: float,
                 chroma_bias: float) -> tuple[np.ndarray, np.ndarray]:
    """The (blocks, 3) mean luma, Cb and Cr of every block of the luma and the chroma noise grids,
    from three word-packed planes (uint32 words)."""
    cw, ch = -(-width // (1 << shift_x)), -(-height // (1 << shift_y))
    nl = -(-width // 16) * -(-height // 16)
    nc = -(-cw // 16) * -(-ch // 16)
    lm, cm = np.zeros(nl * 3, np.float32), np.zeros(nc * 3, np.float32)
    planes = [np.ascontiguousarray(p).view(np.uint32).reshape(-1) for p in (luma, cb, cr)]
    _colour_lib().orc_colour_means(*[p.ctypes.data_as(_u32p) for p in planes], width, height, shift_x, shift_y,
                                   samples_per_word, int(is_float), eight_bit_scale, chroma_bias, _f(lm), _f(cm))
    return lm.reshape(-1, 3), cm.reshape(-1, 3)


def colour_accumulate(records: np.ndarray, means: np.ndarray, width: int, height: int, channels: int, luma: bool,
                      grain_scale: float) -> np.ndarray:
    """One frame's fixed-point cell sums (int32, colour_records x 69 words)."""
    out = np.zeros(colour_records(channels, luma) * COLOUR_CELL_WORDS, np.int32)
    _colour_lib().orc_colour_accumulate(_f(np.ascontiguousarray(records, np.float32)),
                                        _f(np.ascontiguousarray(means, np.float32).reshape(-1)), width, height,
                                        channels, int(luma), grain_scale, out.ctypes.data_as(_i32p))
    return out


def colour_window(ring: np.ndarray, capacity: int, first: int, last: int) -> np.ndarray:
    """The window's decoded sums of frames first..=last from a (capacity, words) int32 ring."""
    ring = np.ascontiguousarray(ring, np.int32).reshape(capacity, -1)
    words = ring.shape[1]
    out = np.zeros(words, np.float32)
    _colour_lib().orc_colour_window(ring.ctypes.data_as(_i32p), capacity, first, last, words, _f(out))
    return out


def colour_levels(window: np.ndarray, ceilings: np.ndarray, cells: int, mean_level: bool) -> np.ndarray:
    out = np.zeros(cells * 2, np.float32)
    _colour_lib().orc_colour_levels(_f(np.ascontiguousarray(window, np.float32)),
                                    _f(np.ascontiguousarray(ceilings, np.float32)), cells, int(mean_level), _f(out))
    return out.reshape(-1, 2)


def colour_fit(window: np.ndarray, planes: int, luma: bool, curve=None, curve_valid: bool = False):
    """Both fits and the gains of the window's sums: (log grain tables, log gain tables, fit headers),
    each plane after plane."""
    table = np.zeros(planes * COLOUR_CELLS, np.float32)
    gains = np.zeros(planes * COLOUR_CELLS, np.float32)
    headers = np.zeros(planes * COLOUR_FIT_PLANE_WORDS, np.float32)
    c = np.ascontiguousarray(curve if curve is not None else np.zeros(16), np.float32)
    _colour_lib().orc_colour_fit(_f(np.ascontiguousarray(window, np.float32)), planes, int(luma), _f(c),
                                 int(curve_valid), _f(table), _f(gains), _f(headers))
    return table, gains, headers


def colour_lookup(table: np.ndarray, colours: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The table's interpolated value and its exponential at each (luma, cb, cr) colour."""
    colours = np.ascontiguousarray(colours, np.float32).reshape(-1, 3)
    values = np.zeros(len(colours), np.float32)
    gains = np.zeros(len(colours), np.float32)
    _colour_lib().orc_colour_lookup(_f(np.ascontiguousarray(table, np.float32)), _f(colours), len(colours),
                                    _f(values), _f(gains))
    return values, gains
