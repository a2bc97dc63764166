"""Pins the CPU oracle's NLMeans restatement to the reference's own host formulas and behavioural
suites (no GPU). Each test names the reference test or formula it re-states."""

import math

import numpy as np
import pytest


def test_h2_inv_norm_formula(oracle):
    # nlmeans/params.rs:229-233: 255^2 / (3 * strength^2 * (2s+1)^2).
    for strength, s in [(1.2, 4), (12.0, 3), (8.0, 2), (0.5, 0)]:
        area = (2 * s + 1) ** 2
        want = np.float32(65025.0) / (np.float32(3.0) * np.float32(strength) * np.float32(strength) * np.float32(area))
        assert oracle.h2_inv_norm(strength, s) == pytest.approx(float(want), rel=1e-7)


def test_welsch_weight_matches_host_formula(oracle):
    # nlmeans/kernels/tests/separable.rs:13-28: host_welsch with H2_INV_NORM 0.6, NOISE_OFFSET 1.13.
    h2, off = 0.6, 1.13
    for total in [0.0, 0.5, 1.13, 1.5, 3.7, 10.0, 40.0]:
        excess = max(total - off, 0.0)
        want = math.exp(-excess * h2)
        got = oracle.welsch_weight(total, h2, off)
        assert got == pytest.approx(want, rel=1e-5)
    assert oracle.welsch_weight(0.5, h2, off) == 1.0  # below the offset: full weight


def test_uniform_image_passthrough(oracle):
    # nlmeans/tests/spatial.rs:5-31: a uniform 0.5 frame stays 0.5 (d=0, a=2, s=2, strength 1.2).
    f = np.full((16, 16, 1), 0.5, np.float32)
    out = oracle.nlm_frame([f], 0, 2, 2, oracle.h2_inv_norm(1.2, 2))
    assert np.abs(out - 0.5).max() < 1e-5


def test_uniform_chroma_passthrough(oracle):
    # nlmeans/tests/spatial.rs:33-64.
    f = np.full((16, 16, 2), 0.5, np.float32)
    out = oracle.nlm_frame([f], 0, 2, 2, oracle.h2_inv_norm(1.2, 2))
    assert out.shape == (16, 16, 2)
    assert np.abs(out - 0.5).max() < 1e-5


def test_noisy_region_suppressed(oracle):
    # nlmeans/tests/spatial.rs:66-98: one bright pixel is pulled toward its flat surround.
    f = np.full((32, 32, 1), 0.5, np.float32)
    f[16, 16, 0] = 0.8
    out = oracle.nlm_frame([f], 0, 3, 1, oracle.h2_inv_norm(50.0, 1))
    assert out[16, 16, 0] < 0.8


def test_high_strength_smooths_heavily(oracle):
    # nlmeans/tests/spatial.rs:100+: at strength 10000 a checkerboard averages toward its mean.
    f = np.zeros((16, 16, 1), np.float32)
    f[::2, ::2] = 1.0
    f[1::2, 1::2] = 1.0
    out = oracle.nlm_frame([f], 0, 2, 1, oracle.h2_inv_norm(10000.0, 1))
    inner = out[4:12, 4:12, 0]
    assert np.abs(inner - 0.5).max() < 0.15


def test_strength_monotonic(oracle):
    rng = np.random.default_rng(5)
    f = np.clip(0.5 + 0.1 * rng.standard_normal((24, 24, 1)), 0, 1).astype(np.float32)
    prev = None
    for strength in [1.0, 4.0, 16.0]:
        out = oracle.nlm_frame([f], 0, 2, 1, oracle.h2_inv_norm(strength, 1))
        dev = float(np.abs(out - f).mean())
        if prev is not None:
            assert dev > prev
        prev = dev


def test_transpose_symmetry(oracle):
    # Transposing the frame transposes the result (the window and patch are square).
    rng = np.random.default_rng(7)
    f = rng.random((20, 20, 1), dtype=np.float32)
    h2 = oracle.h2_inv_norm(20.0, 2)
    a = oracle.nlm_frame([f], 0, 2, 2, h2)
    b = oracle.nlm_frame([np.ascontiguousarray(f.transpose(1, 0, 2))], 0, 2, 2, h2)
    np.testing.assert_allclose(a, b.transpose(1, 0, 2), rtol=0, atol=2e-6)


def test_temporal_static_scene_equals_repeat(oracle):
    # With d=1 and three identical frames the pair passes see the same content as the centre.
    rng = np.random.default_rng(3)
    f = rng.random((16, 20, 1), dtype=np.float32)
    h2 = oracle.h2_inv_norm(10.0, 1)
    out = oracle.nlm_frame([f, f, f], 1, 2, 1, h2)
    assert np.isfinite(out).all()
    assert np.abs(out - f).mean() < np.abs(f - f.mean()).mean()


def test_fp32_mirror_tracks_fp64(oracle):
    rng = np.random.default_rng(11)
    frames = [rng.random((24, 28, 2), dtype=np.float32) for _ in range(3)]
    h2 = oracle.h2_inv_norm(30.0, 2)
    a = oracle.nlm_frame(frames, 1, 3, 2, h2)
    b = oracle.nlm_frame(frames, 1, 3, 2, h2, fp64=True)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    assert rel.max() < 1e-5


def test_egress_rounds_half_up_and_clamps(oracle):
    # engine/kernels.rs:133-134: u32(clamp(v,0,1) * max + 0.5).
    fr = np.array([[-0.2, 0.0, 0.5 / 255, 1.5 / 255, 1.0, 1.7]], np.float32).reshape(1, 6, 1)
    (codes,) = oracle.egress(fr, 0, 255.0)
    assert codes.tolist() == [[0, 0, 1, 2, 255, 255]]


def test_ingest_egress_round_trip_all_depths(oracle):
    rng = np.random.default_rng(0)
    for kind, depth in [(0, 8), (1, 10), (1, 12), (1, 16)]:
        maxc = (1 << depth) - 1
        y = rng.integers(0, maxc + 1, (7, 9)).astype(np.uint8 if depth == 8 else np.uint16)
        u = rng.integers(0, maxc + 1, (7, 9)).astype(y.dtype)
        fr = oracle.ingest([y, u], kind, float(maxc))
        back = oracle.egress(fr, kind, float(maxc))
        assert np.array_equal(back[0], y) and np.array_equal(back[1], u)


def test_f32_ingest_bias(oracle):
    # engine/kernels.rs:64-90 / 159-184: chroma float samples are biased by +0.5 on the way in.
    y = np.array([[-0.25, 0.25]], np.float32)
    fr = oracle.ingest([y, y], 2, 1.0, bias=0.5)
    assert fr[0, :, 0].tolist() == [0.25, 0.75]
    back = oracle.egress(fr, 2, 1.0, bias=0.5)
    assert back[0].tolist() == [[-0.25, 0.25]]


def test_stream_repeat_edges(oracle):
    # ring.rs:103-146: the first and last frames repeat at the stream edges.
    rng = np.random.default_rng(2)
    frames = [rng.random((12, 12, 1), dtype=np.float32) for _ in range(3)]
    h2 = oracle.h2_inv_norm(10.0, 1)
    outs = oracle.nlm_stream_repeat(frames, 2, 1, 1, h2)
    first = oracle.nlm_frame([frames[0], frames[0], frames[0], frames[1], frames[2]], 2, 1, 1, h2)
    assert np.array_equal(outs[0], first)
    last = oracle.nlm_frame([frames[0], frames[1], frames[2], frames[2], frames[2]], 2, 1, 1, h2)
    assert np.array_equal(outs[2], last)


# ---- motion compensation (motion/kernels/compensate.rs, nlmeans/dispatch/motion.rs) ---------------

def test_mc_warp_follows_each_blocks_vector(oracle):
    rng = np.random.default_rng(1)
    f = rng.random((20, 28, 2), dtype=np.float32)
    bx, by, step = 4, 3, 8
    assert np.array_equal(oracle.mc_warp(f, np.zeros((bx * by, 2), np.int32), step, bx, by), f)
    mv = np.zeros((bx * by, 2), np.int32)
    mv[:] = (2, -1)
    got = oracle.mc_warp(f, mv, step, bx, by)
    ys, xs = np.mgrid[0:20, 0:28]
    assert np.array_equal(got, f[np.clip(ys - 1, 0, 19), np.clip(xs + 2, 0, 27)])
    mv[bx * by - 1] = (-5, 4)  # the last block also covers the ragged right and bottom edges
    got = oracle.mc_warp(f, mv, step, bx, by)
    assert np.array_equal(got[16:, 24:], f[np.clip(ys[16:, 24:] + 4, 0, 19), np.clip(xs[16:, 24:] - 5, 0, 27)])


@pytest.mark.parametrize("d,chained", [(1, False), (2, False), (3, True)])
def test_motion_compensation_of_a_still_clip_is_the_plain_pass(oracle, d, chained):
    """Every block of identical frames matches where it stands, so the warped window is the window
    and the output is the plain pass's, bit for bit."""
    rng = np.random.default_rng(2)
    f = rng.random((40, 48, 1), dtype=np.float32)
    frames = [f] * 4
    h2 = oracle.h2_inv_norm(6.0, 1)
    plain = oracle.nlm_stream_repeat(frames, d, 2, 1, h2)
    mc = oracle.nlm_stream_mc(frames, d, 2, 1, h2, chained=chained)
    assert all(np.array_equal(x, y) for x, y in zip(plain, mc))


def test_exp_mirror_within_one_ulp(oracle):
    # The FP32 mirror's exponential (nlm_oracle.cpp `exp_mirror`) against the double-precision
    # exponential over the weights' whole range: within 1 ulp everywhere, exact at 0, and 0 below -87.
    x = np.concatenate([np.linspace(-87.0, 0.0, 2_000_003, dtype=np.float32),
                        -np.geomspace(1e-8, 1.0, 100_001).astype(np.float32),
                        np.linspace(0.0, 88.0, 200_001, dtype=np.float32)])
    got = oracle.exp_mirror(x).astype(np.float64)
    want = np.exp(x.astype(np.float64))
    ulp = np.spacing(want.astype(np.float32)).astype(np.float64)
    err = np.abs(got - want) / ulp
    assert err.max() <= 1.0, float(err.max())
    assert oracle.exp_mirror(np.array([0.0, -0.0, -87.5, np.nan], np.float32)).tolist() == [1.0, 1.0, 0.0, 0.0]
