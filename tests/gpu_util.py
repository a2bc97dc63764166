"""Helpers for the GPU tests: drive an engine through the C ABI with torch device buffers, and
compute the oracle's result for the same stream."""

from __future__ import annotations

import numpy as np

from conftest import avd


def to_words(codes: np.ndarray, fmt) -> np.ndarray:
    flat = codes.reshape(-1)
    if fmt.kind == 2:
        return np.ascontiguousarray(flat.astype(np.float32))
    spw = fmt.samples_per_word()
    pad = (-flat.size) % spw
    dt = np.uint8 if fmt.kind == 0 else np.uint16
    return np.ascontiguousarray(np.concatenate([flat.astype(dt), np.zeros(pad, dt)])).view(np.uint32)


def from_words(words: np.ndarray, fmt, w: int, h: int) -> np.ndarray:
    if fmt.kind == 2:
        return words.view(np.float32)[: w * h].reshape(h, w).copy()
    dt = np.uint8 if fmt.kind == 0 else np.uint16
    return words.view(dt)[: w * h].reshape(h, w).copy()


class Runner:
    """Pushes a clip through an engine and collects every emitted frame on the host."""

    def __init__(self, spec, tuning=None):
        import torch

        self.torch = torch
        self.spec = spec
        self.geometry = spec.geometry
        self.engine = avd.build_engine(spec, tuning)
        self.stream = torch.cuda.current_stream()
        self.engine.set_stream(self.stream.cuda_stream)
        g = self.geometry
        self.dims = [g.plane_dims(i) for i in range(g.plane_count())]
        self.out_bufs = [self._alloc(g.output, w, h, fill=0x5A5A5A5A) for (w, h) in self.dims]

    def _alloc(self, fmt, w, h, fill=0):
        t = self.torch
        words = fmt.plane_bytes(w * h) // 4
        buf = t.full((words,), fill, dtype=t.int64, device="cuda").to(t.int32) if fill else t.zeros(
            words, dtype=t.int32, device="cuda")
        return buf

    def planes_for(self, frame: list[np.ndarray], fmt):
        t = self.torch
        bufs, planes = [], []
        for (w, h), codes in zip(self.dims, frame):
            words = to_words(codes, fmt)
            buf = t.from_numpy(words.view(np.int32).copy()).to("cuda")
            bufs.append(buf)
            planes.append(avd.DevicePlane.from_tensor(buf, w, h))
        return bufs, planes

    def out_planes(self):
        return [avd.DevicePlane.from_tensor(b, w, h) for b, (w, h) in zip(self.out_bufs, self.dims)]

    def emit(self) -> list[np.ndarray]:
        self.engine.emit_into(self.out_planes())
        self.torch.cuda.synchronize()
        g = self.geometry
        res = []
        for b, (w, h) in zip(self.out_bufs, self.dims):
            words = b.cpu().numpy().view(np.uint32)
            res.append(from_words(words, g.output, w, h))
            if g.output.kind != 2:
                # engine/plane.rs:265-269: the padding past the last sample is written as zeros.
                spw = g.output.samples_per_word()
                pad = (-(w * h)) % spw
                if pad:
                    dt = np.uint8 if g.output.kind == 0 else np.uint16
                    tail = words.view(dt)[w * h:w * h + pad]
                    assert not tail.any(), "output padding must be zero"
        return res

    def run(self, clip: list[list[np.ndarray]], context: int = 0) -> list[list[np.ndarray]]:
        outs = []
        keep = []
        for i, frame in enumerate(clip):
            bufs, planes = self.planes_for(frame, self.geometry.input)
            keep.append(bufs)
            if i < context:
                self.engine.push_context(planes)
                continue
            ready = self.engine.push(planes)
            for _ in range(ready):
                outs.append(self.emit())
        tail = self.engine.finish()
        for _ in range(tail):
            outs.append(self.emit())
        return outs


def hq_fixed_words(strength: float, sigma: float, s: int, channels: int, a: int):
    """h2, the noise offset and the spatial offset table of NLMeans-HQ with a pinned sigma, in the
    reference's f32 arithmetic (nlmeans/params.rs:221-268, noise/correlation.rs:43-88 at rho 0)."""
    f = np.float32
    area = f((2 * s + 1) ** 2)
    eff = f(strength) * f(sigma) * f(255.0)
    h2 = f(65025.0) / (((f(3.0) * eff) * eff) * area)
    scale = f(3.0) if channels == 1 else f(1.5)
    sum_sq = f(0.0)
    for _ in range(channels):
        sum_sq = f(sum_sq + f(sigma) * f(sigma))
    offset = ((f(2.0) * scale) * sum_sq) * area
    side = 2 * a + 1
    lut = np.full(side * side, offset, np.float32)
    lut[a * side + a] = 0.0
    return float(h2), float(offset), lut


def oracle_pass(oracle, frames: list[list[np.ndarray]], fmt, d, a, s, strength, wref=1.0, chroma=False,
                out_fmt=None, exact=False, hq_sigma=None, hq_confidence=False, thsad_scale=1.0, prefilter=None,
                motion=None, share_writes=None, share_reads=None):
    """The oracle's output planes for one plane group over a stream (repeat edges).

    `prefilter` is an `avd.PrefilterMode` (or None); `motion` an `avd.MotionSearch` for motion
    compensation (or None). Returns the FP32-mirror output planes; with `exact`, also the FP64
    outputs as (H, W, C) normalised floats, which mark the samples that sit on a rounding tie."""
    out_fmt = out_fmt or fmt
    bias = 0.5 if (chroma and fmt.kind == 2) else 0.0
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), bias) for p in frames]
    h2, off, lut = oracle.h2_inv_norm(strength, s), 0.0, None
    if hq_sigma is not None:
        h2, off, lut = hq_fixed_words(strength, hq_sigma, s, 2 if chroma else 1, a)
    pf = None
    if prefilter is not None and prefilter.kind == 1:
        pf = ("bilateral", prefilter.sigma_s, prefilter.sigma_r)
    elif prefilter is not None and prefilter.kind == 2:
        # nlmeans/denoiser/noise.rs:343-390: the pilot runs at h2 / scale^2 with the input's offset
        # table; the main pass compares pilot outputs with no offset at all.
        pf = ("nlm", oracle.pilot_h2(h2, prefilter.strength_scale), lut)
        off, lut = 0.0, None
    cs = hq_sigma if hq_confidence else None
    if motion is not None and d > 0:
        # nlmeans/denoiser/noise.rs:360-363: the window search's floor at the pinned sigma times the
        # prefilter's residual fraction (0 for both prefilters).
        sigma_y = (hq_sigma or 0.0) * (0.0 if pf is not None else 1.0)
        chained = motion.estimation == avd.MotionEstimation.CHAINED or (
            motion.estimation == avd.MotionEstimation.AUTO and d >= 3)
        refine = motion.refine_radius if motion.estimation == avd.MotionEstimation.CHAINED else 2

        def run(fp64):
            return oracle.nlm_stream_mc(f32, d, a, s, h2, wref=wref, noise_offset=off, lut=lut,
                                        confidence=hq_confidence, sad_floor=oracle.sad_noise_floor(motion.blksize,
                                                                                                   sigma_y),
                                        thsad_scale=thsad_scale, blksize=motion.blksize, overlap=motion.overlap,
                                        search_radius=motion.search_radius, levels=motion.pyramid_levels,
                                        chained=chained, refine_radius=refine, prefilter=pf, fp64=fp64,
                                        share_writes=None if fp64 else share_writes, share_reads=share_reads,
                                        ceiling=motion.max_search_escalation
                                        if motion.max_search_escalation > motion.search_radius else 0)
    else:
        def run(fp64):
            return oracle.nlm_stream_repeat(f32, d, a, s, h2, wref=wref, noise_offset=off, lut=lut, fp64=fp64,
                                            conf_sigma=cs, thsad_scale=thsad_scale, prefilter=pf)
    outs = run(False)
    obias = 0.5 if (chroma and out_fmt.kind == 2) else 0.0
    planes = [oracle.egress(o, out_fmt.kind, out_fmt.max_value(), obias) for o in outs]
    if not exact:
        return planes
    return planes, run(True)


# A sample whose exact (FP64) value lies within this distance, in normalised units, of a rounding
# boundary is a tie: any two float32 implementations may round it either way. It is about four
# times the largest float difference seen between the GPU kernel and the FP32 oracle.
TIE_BAND = 4e-6


class Parity:
    """Aggregates GPU-vs-oracle agreement over every frame and plane of a stream.

    The bar is the north-star's: no sample more than 1 LSB apart, and at least 99.9% of all
    samples identical (`identical`, the raw share). Where the exact value sits on a rounding tie
    (an average of two integer codes is a half code; the self weight equals the best match's
    weight, so this happens whenever one neighbour dominates) only the last bit of a float32
    evaluation decides: the engine's exact finish recomputes those samples in the oracle's own
    operation order. The share over the samples that are not ties is reported beside it."""

    def __init__(self):
        self.total = self.same = self.ties = self.same_nontie = self.nontie = 0
        self.max_lsb = 0

    def add(self, got: np.ndarray, want: np.ndarray, exact: np.ndarray | None, max_value: float,
            tie_band: float = TIE_BAND):
        diff = np.abs(got.astype(np.int64) - want.astype(np.int64))
        self.max_lsb = max(self.max_lsb, int(diff.max()) if diff.size else 0)
        self.total += diff.size
        self.same += int((diff == 0).sum())
        if exact is None:
            tie = np.zeros(diff.shape, bool)
        else:
            t = np.clip(exact, 0.0, 1.0) * max_value + 0.5
            tie = np.abs(t - np.rint(t)) < tie_band * max_value
        self.ties += int(tie.sum())
        self.nontie += int((~tie).sum())
        self.same_nontie += int(((diff == 0) & ~tie).sum())

    def stats(self) -> dict:
        return {"samples": self.total, "identical": self.same / max(1, self.total),
                "identical_excluding_ties": self.same_nontie / max(1, self.nontie), "ties": self.ties,
                "max_lsb": self.max_lsb}

    def check(self, min_identical: float = 0.999, min_raw: float = 0.999):
        st = self.stats()
        assert st["max_lsb"] <= 1, st
        assert st["identical_excluding_ties"] >= min_identical, st
        assert st["identical"] >= min_raw, st
        return st


def parity_stats(got: np.ndarray, want: np.ndarray) -> tuple[float, int]:
    diff = np.abs(got.astype(np.int64) - want.astype(np.int64))
    return float((diff == 0).mean()), int(diff.max())


def assert_parity(got: np.ndarray, want: np.ndarray, min_identical: float = 0.999, max_lsb: int = 1):
    ident, mx = parity_stats(got, want)
    assert mx <= max_lsb and ident >= min_identical, f"identical {ident:.6f}, max |diff| {mx} LSB"
