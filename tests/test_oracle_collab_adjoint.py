"""The NL4D Wiener stage and the collab pass's adjoint on the CPU. Neither exists in the reference
(its filter, collab/kernels/fused/mod.rs:559-850, stops at the threshold), so the f64 restatement
(oracle/collab_adjoint_oracle.cpp) is their oracle: its adjoint is checked by central finite
differences of its own forward with the groups and keep decisions held fixed, and its forward
against the f32 restatement's accumulators."""

import numpy as np
import pytest

from collab_cases import cross_frame_setup

POOL_RATIO = 2.42 / 4.158


def adjoint_case(seed: int, channels: int, radius: int, pooled: bool, wiener: bool, w: int = 40, h: int = 32):
    """A pass over textured noisy frames: the f32 restatement's accumulators and records."""
    import oracle

    rng = np.random.default_rng(seed)
    frames = 2 * radius + 1
    y, x = np.mgrid[0:h * frames, 0:w].astype(np.float32)
    planes = [0.5 + 0.2 * np.sin(x * 0.31 + y * 0.13 + k) + rng.normal(0, 0.04, x.shape) for k in range(channels)]
    ring = np.stack(planes, axis=-1).astype(np.float32).reshape(-1)
    case = dict(centre_slot=radius, radius=radius, c_min=0.3, refine=2, spatial_radius=5, k_max=8,
                sigma=tuple(0.04 + 0.01 * k for k in range(channels)), lambda_ht=2.7, kaiser_beta=2.0,
                pooled=POOL_RATIO if pooled else None, wiener=wiener)
    if radius:
        bx, by = -(-w // 8), -(-h // 8)
        case.update(mv_field=rng.integers(-3, 4, 2 * radius * bx * by * 2).astype(np.int32),
                    confidence=rng.uniform(0, 1, 2 * radius * bx * by).astype(np.float32),
                    neighbour_slots=np.array([s for t in range(radius) for s in (radius - 1 - t, radius + 1 + t)],
                                             np.uint32),
                    mv_stride=bx * by * 2, conf_stride=bx * by, blocks_x=bx, blocks_y=by)
    record = {}
    acc, ws, gw = oracle.collab_fused(ring, w, h, channels, record=record, **case)
    return dict(ring=ring, w=w, h=h, channels=channels, case=case, record=record, accum=acc, wsum=ws, gw=gw)


def f64(c, ring=None, sigma=None, grads=None):
    import oracle

    k = c["case"]
    kw = dict(centre_slot=k["centre_slot"], radius=k["radius"], neighbour_slots=k.get("neighbour_slots"),
              wiener=k["wiener"], sigma=sigma)
    if grads is not None:
        kw.update(grad_accum=grads[0], grad_wsum=grads[1])
    return oracle.collab64(c["ring"] if ring is None else ring, c["w"], c["h"], c["channels"], c["record"], **kw)


CASES = [(1, 1, 0, False, False), (2, 1, 2, False, True), (3, 1, 1, True, False), (4, 1, 2, True, True),
         (5, 2, 2, False, True), (6, 2, 1, True, True), (7, 2, 0, False, False)]


@pytest.mark.parametrize("seed,channels,radius,pooled,wiener", CASES)
def test_f64_forward_is_the_f32_pass(oracle, seed, channels, radius, pooled, wiener):
    """Over the recorded groups and masks the f64 forward is the f32 pass up to rounding: the
    normalised frames agree to 5e-3 on every covered pixel. (The f32 pass rounds every weight
    contribution to 1 / (5 accum_scale), about 3e-6 at radius 2, against contributions of a few
    hundredths of a percent of the Kaiser-tapered group weight, hence the tolerance.)"""
    c = adjoint_case(seed, channels, radius, pooled, wiener)
    a64, w64 = f64(c)
    cov = c["wsum"] > 0
    assert np.array_equal(cov, w64 > 0)
    out32 = c["accum"].reshape(-1, channels)[cov] * 5.0 / c["wsum"][cov, None]
    out64 = a64.reshape(-1, channels)[cov] / w64[cov, None]
    assert np.abs(out32 - out64).max() < 5e-3
    assert np.abs(out32 - out64).mean() < 2e-4
    scale = oracle.cross_frame_accum_scale(c["case"]["spatial_radius"], radius)
    assert np.abs(c["wsum"] / (5 * scale) - w64).max() <= 1e-4 * w64.max()


@pytest.mark.parametrize("seed,channels,radius,pooled,wiener", CASES)
def test_f64_adjoint_matches_central_differences(oracle, seed, channels, radius, pooled, wiener):
    """L = <gA, A> + <gW, W>: the adjoint's dL/d(ring) at 16 sampled samples and dL/d(sigma_c)
    agree with central differences (step 1e-6, 1e-7 for sigma) to 1e-4 relative."""
    c = adjoint_case(seed, channels, radius, pooled, wiener)
    rng = np.random.default_rng(100 + seed)
    a64, w64 = f64(c)
    ga, gw = rng.normal(0, 1, a64.shape), rng.normal(0, 1, w64.shape)
    grad_ring, grad_sigma = f64(c, grads=(ga, gw))

    def loss(ring=None, sigma=None):
        a, w = f64(c, ring=ring, sigma=sigma)
        return float((ga * a).sum() + (gw * w).sum())

    ring = c["ring"].astype(np.float64)
    touched = np.flatnonzero(grad_ring)
    assert touched.size > 0
    eps = 1e-6
    for i in rng.choice(touched, 16, replace=False):
        up, down = ring.copy(), ring.copy()
        up[i] += eps
        down[i] -= eps
        fd = (loss(ring=up) - loss(ring=down)) / (2 * eps)
        assert abs(fd - grad_ring[i]) <= 1e-4 * max(abs(grad_ring[i]), 1e-2), (i, fd, grad_ring[i])
    sig = np.asarray(c["record"]["sigma"], np.float64)
    for ch in range(channels):
        up, down = sig.copy(), sig.copy()
        up[ch] += 1e-7
        down[ch] -= 1e-7
        fd = (loss(sigma=up) - loss(sigma=down)) / 2e-7
        assert abs(fd - grad_sigma[ch]) <= 1e-4 * max(abs(grad_sigma[ch]), 1.0), (ch, fd, grad_sigma[ch])


def test_hard_threshold_output_does_not_depend_on_sigma(oracle):
    """With the keep masks fixed and no Wiener stage a group's retained variance and its weight-scale
    word both move as sigma_0^2, so no group weight moves with sigma and the normalised frame A / W
    has a zero sigma gradient (so do A and W on their own); the Wiener gains make it nonzero."""
    for wiener in (False, True):
        c = adjoint_case(11, 1, 1, False, wiener)
        a64, w64 = f64(c)
        cov = w64 > 0
        out = np.zeros_like(a64)
        out[cov] = a64[cov] / w64[cov]
        g = np.random.default_rng(3).normal(0, 1, a64.shape) * cov
        # d(A/W): dA = g / W, dW = -g A / W^2.
        ga = np.where(cov, g / np.where(cov, w64, 1), 0)
        gw = np.where(cov, -g * out / np.where(cov, w64, 1), 0)
        _, grad_sigma = f64(c, grads=(ga, gw))
        # Here the Wiener gradient is about 1.6 and the hard threshold's f64 rounding, 1e-14.
        if wiener:
            assert abs(grad_sigma[0]) > 0.1
        else:
            assert abs(grad_sigma[0]) < 1e-9
            rng = np.random.default_rng(4)
            _, alone = f64(c, grads=(rng.normal(0, 1, a64.shape), rng.normal(0, 1, w64.shape)))
            assert abs(alone[0]) < 1e-9


def test_wiener_stage_shrinks_kept_coefficients(oracle):
    """The Wiener pass keeps the same groups and masks and moves the output towards the group
    means: on a flat noisy field its residual variance is below the hard threshold's."""
    case = cross_frame_setup(48, 40, 1)
    rng = np.random.default_rng(5)
    ring = (np.full(case.pop("ring").shape, 0.5) + rng.normal(0, 0.05, (48 * 40 * 3,))).astype(np.float32)
    w, h = case.pop("width"), case.pop("height")
    case.pop("channels")
    case.update(sigma=(0.05,), lambda_ht=2.7, kaiser_beta=2.0)
    outs = {}
    for wiener in (False, True):
        rec = {}
        acc, ws, _ = oracle.collab_fused(ring, w, h, 1, wiener=wiener, record=rec, **case)
        sl = slice(w * h, 2 * w * h)
        outs[wiener] = acc[sl] * 5.0 / ws[sl]
        if wiener:
            assert np.array_equal(rec["members"], hard_rec["members"])
            # A kept coefficient stays kept: the stage scales, it never zeroes.
            assert np.array_equal(rec["masks"], hard_rec["masks"])
        else:
            hard_rec = rec
    assert np.var(outs[True] - 0.5) < np.var(outs[False] - 0.5)
