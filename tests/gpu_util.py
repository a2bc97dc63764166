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

    def __init__(self, spec):
        import torch

        self.torch = torch
        self.spec = spec
        self.geometry = spec.geometry
        self.engine = avd.build_engine(spec)
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


def oracle_pass(oracle, frames: list[list[np.ndarray]], fmt, d, a, s, strength, wref=1.0, chroma=False,
                out_fmt=None):
    """The oracle's output planes for one plane group over a stream (repeat edges)."""
    out_fmt = out_fmt or fmt
    bias = 0.5 if (chroma and fmt.kind == 2) else 0.0
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), bias) for p in frames]
    h2 = oracle.h2_inv_norm(strength, s)
    outs = oracle.nlm_stream_repeat(f32, d, a, s, h2, wref=wref)
    obias = 0.5 if (chroma and out_fmt.kind == 2) else 0.0
    return [oracle.egress(o, out_fmt.kind, out_fmt.max_value(), obias) for o in outs]


def parity_stats(got: np.ndarray, want: np.ndarray) -> tuple[float, int]:
    diff = np.abs(got.astype(np.int64) - want.astype(np.int64))
    return float((diff == 0).mean()), int(diff.max())


def assert_parity(got: np.ndarray, want: np.ndarray, min_identical: float = 0.999, max_lsb: int = 1):
    ident, mx = parity_stats(got, want)
    assert mx <= max_lsb and ident >= min_identical, f"identical {ident:.6f}, max |diff| {mx} LSB"
