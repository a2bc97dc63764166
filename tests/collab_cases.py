"""Inputs of the reference's recorded NL4D group-filter cases, rebuilt from their closed-form
definitions (av-denoise-core/src/collab/tests/helpers.rs:10-55 and collab/tests/fused/mod.rs:55-
733), and the digest the reference takes of a run (fused/mod.rs:187-301)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = json.loads((Path(__file__).parent / "golden" / "collab_recorded.json").read_text())

BLKSIZE, BLK_STEP = 16, 8
DIGEST_RELATIVE_TOLERANCE = 2.0e-5  # fused/mod.rs:283
PROBE_TOLERANCE = 1.0e-3  # fused/mod.rs:290


def _hash(idx: np.ndarray) -> np.ndarray:
    h = (idx.astype(np.uint64) * np.uint64(2654435761) + np.uint64(0x9E3779B9)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(15)
    h = (h * np.uint64(0x85EBCA6B)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    return h.astype(np.uint32)


def _unit(h: np.ndarray) -> np.ndarray:
    return h.astype(np.float32) / np.float32(4294967295.0)


def make_unique_frame(width: int, height: int) -> np.ndarray:
    """helpers.rs:36-53: a horizontal ramp plus a per-pixel hash offset."""
    idx = np.arange(width * height, dtype=np.uint64)
    offset = _unit(_hash(idx))
    x = (np.arange(width * height) % width).astype(np.float32)
    return (x * np.float32(10.0) + offset * np.float32(10.0)).astype(np.float32)


def unique_frame(width: int, height: int) -> np.ndarray:
    """fused/mod.rs:60-64: the unique frame divided by its peak."""
    raw = make_unique_frame(width, height)
    return (raw / raw.max()).astype(np.float32)


def noisy_flat_field(width: int, height: int, base: float, sigma: float) -> np.ndarray:
    """helpers.rs:10-27: Irwin-Hall noise from four hashed uniforms per sample."""
    unit_std = np.sqrt(np.float32(1.0) / np.float32(3.0)).astype(np.float32)
    idx = np.arange(width * height, dtype=np.uint64)
    total = np.zeros(width * height, np.float32)
    for k in range(4):
        total = (total + (_unit(_hash(idx * np.uint64(4) + np.uint64(k))) - np.float32(0.5))).astype(np.float32)
    return (np.float32(base) + (total / unit_std) * np.float32(sigma)).astype(np.float32)


def spatial_only(frame: np.ndarray, width: int, height: int, **over) -> dict:
    case = dict(ring=frame, width=width, height=height, channels=1, centre_slot=0, radius=0, c_min=0.0,
                refine=0, spatial_radius=4, k_max=8, sigma=(0.02,), lambda_ht=5.3, rho=0.0, kaiser_beta=0.0)
    case.update(over)
    return case


def cross_frame_setup(width: int, height: int, radius: int) -> dict:
    """fused/mod.rs:586-637."""
    frames = 2 * radius + 1
    blocks_x, blocks_y = -(-width // BLK_STEP), -(-height // BLK_STEP)
    conf_stride = blocks_x * blocks_y
    mv_stride = conf_stride * 2
    mv = np.zeros(2 * radius * mv_stride, np.int32)
    conf = np.zeros(2 * radius * conf_stride, np.float32)
    for t in range(2 * radius):
        for block in range(conf_stride):
            i = t * mv_stride + block * 2
            mv[i] = (block % 11) - 5 + t
            mv[i + 1] = 4 - (block % 9) - t
            conf[t * conf_stride + block] = np.float32(((block * 7 + t * 3) % 11)) / np.float32(10.0)
    slots = []
    for t in range(radius):
        slots += [radius - 1 - t, radius + 1 + t]
    return spatial_only(unique_frame(width, height * frames), width, height, mv_field=mv, confidence=conf,
                        neighbour_slots=np.array(slots, np.uint32), centre_slot=radius, c_min=0.5, radius=radius,
                        refine=2, mv_stride=mv_stride, conf_stride=conf_stride, blocks_x=blocks_x,
                        blocks_y=blocks_y)


def five_frame_ring_with_jittered_copies(width: int, height: int) -> dict:
    """fused/mod.rs:689-732."""
    radius = 2
    frame = unique_frame(width, height)
    jitter = noisy_flat_field(width, height * 4, 0.5, 0.002)
    pixels = width * height
    ring = []
    for slot in range(5):
        if slot == radius:
            ring.append(frame)
            continue
        n = slot if slot < radius else slot - 1
        ring.append(((frame + jitter[n * pixels:(n + 1) * pixels]).astype(np.float32) - np.float32(0.5)).astype(
            np.float32))
    blocks_x, blocks_y = -(-width // BLK_STEP), -(-height // BLK_STEP)
    conf_stride = blocks_x * blocks_y
    mv_stride = conf_stride * 2
    return spatial_only(np.concatenate(ring), width, height, mv_field=np.zeros(2 * radius * mv_stride, np.int32),
                        confidence=np.ones(2 * radius * conf_stride, np.float32),
                        neighbour_slots=np.array([0, 1, 3, 4], np.uint32), centre_slot=radius, radius=radius,
                        refine=0, mv_stride=mv_stride, conf_stride=conf_stride, blocks_x=blocks_x,
                        blocks_y=blocks_y)


def recorded_cases() -> dict[str, dict]:
    """collab/tests/fused/recorded.rs: every recorded case's inputs, by label."""
    u = unique_frame(128, 96)
    t = unique_frame(96, 128).reshape(128, 96).T.copy().reshape(-1)
    noise = noisy_flat_field(64, 64, 0.5, 0.05)
    return {
        "unique content": spatial_only(u, 128, 96),
        "transposed ramp": spatial_only(t, 128, 96),
        "ragged reference row": spatial_only(unique_frame(104, 96), 104, 96),
        "short search space": spatial_only(unique_frame(64, 64), 64, 64, spatial_radius=1),
        "noise": spatial_only(noise, 64, 64),
        "correlation shaping": spatial_only(noise, 64, 64, rho=0.86),
        "cross frame": cross_frame_setup(64, 64, 2),
        "planted cross-frame match": five_frame_ring_with_jittered_copies(64, 64),
    }


def digest(accum: np.ndarray, wsum: np.ndarray, group_weight: np.ndarray) -> dict:
    """fused/mod.rs:221-259 for a luma run: covered pixels, mean, RMS, mean group weight, probes."""
    a = accum.astype(np.float64)
    w = wsum.astype(np.float64)
    pix = np.where(wsum != 0, a * 5.0 / np.where(wsum != 0, w, 1.0), 0.0)
    n = pix.size
    probes = [float(pix[(i * 7919 + 1013) % n]) for i in range(8)]
    return {"covered": int((wsum != 0).sum()), "pixel_mean": float(pix.sum() / n),
            "pixel_rms": float(np.sqrt((pix * pix).sum() / n)),
            "weight_mean": float(group_weight.astype(np.float64).mean()), "probes": probes}


def assert_matches_recorded(label: str, got: dict, want: dict) -> None:
    """fused/mod.rs:304-330."""
    assert got["covered"] == want["covered"], (label, got["covered"], want["covered"])
    for k in ("pixel_mean", "pixel_rms", "weight_mean"):
        rel = abs(got[k] - want[k]) / max(abs(want[k]), 1e-30)
        assert rel < DIGEST_RELATIVE_TOLERANCE, (label, k, got[k], want[k], rel)
    for i, (g, e) in enumerate(zip(got["probes"], want["probes"])):
        assert abs(g - e) < PROBE_TOLERANCE, (label, i, g, e)
