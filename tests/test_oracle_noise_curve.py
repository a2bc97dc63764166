"""The oracle's noise curve and luma quarter fields on the CPU.

The reading cases replay noise/tests/curve.rs (av-denoise-core): the populated bin counts and the
curve flags it asserts, and its check that the curve agrees with the host model within 2 ulp
(noise/curve.rs:71-235, restated in noise_curve_cases.host_curve). The quarter-field cases check the
stats restatement against direct numpy sums on real frames.
"""

import numpy as np
import pytest

import noise_curve_cases as cc

R_VALID, R_CURVE_VALID, R_QUARTER_MEDIAN, R_POPULATED, R_RATIOS = 2, 11, 12, 13, 14


def reading(o, frame, records=None, curve=True):
    rec = frame.records() if records is None else records
    return o.noise_reading(rec, [0.01, 0.0], 1, frame.w, frame.h, True, curve)


@pytest.mark.parametrize("name,build,populated,has_curve", cc.CASES, ids=[c[0] for c in cc.CASES])
def test_reference_curve_cases(name, build, populated, has_curve):
    import oracle as o

    frame = build()
    records = frame.records()
    r = reading(o, frame, records)
    assert int(r[R_POPULATED]) == populated
    assert bool(r[R_CURVE_VALID]) == has_curve
    host = cc.host_curve(frame, records)
    if not has_curve:
        assert not r[R_RATIOS:].any() and r[R_QUARTER_MEDIAN] == 0
        return
    assert host is not None
    median, ratios = host
    assert cc.ulp_gap(r[R_QUARTER_MEDIAN], median) <= 2
    for b in range(16):
        assert cc.ulp_gap(r[R_RATIOS + b], ratios[b]) <= 2, (b, r[R_RATIOS + b], ratios[b])


def test_the_curve_rises_with_the_bins():
    import oracle as o

    r = reading(o, cc.case_bins(3))
    assert r[R_RATIOS + 15] > r[R_RATIOS]
    # Flat before the first populated bin (1) and past the last (13).
    assert r[R_RATIOS] == r[R_RATIOS + 1] and r[R_RATIOS + 15] == r[R_RATIOS + 13]


def test_a_32nd_quarter_populates_the_bin_and_raises_its_ratio():
    import oracle as o

    empty = reading(o, cc.case_bin_count(31))
    full = reading(o, cc.case_bin_count(32))
    assert full[R_RATIOS + 4] > empty[R_RATIOS + 4]


def test_curve_off_writes_zero_curve_words():
    import oracle as o

    frame = cc.case_bins(3)
    r = reading(o, frame, curve=False)
    assert r[R_VALID] == 1.0
    assert not r[R_CURVE_VALID:].any()


def _frames(w, h, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = (0.5 + 0.4 * np.sin(x * 0.05) * np.cos(y * 0.04)).astype(np.float32)[..., None]
    a = np.clip(base + rng.normal(0, 4 / 255, base.shape), 0, 1).astype(np.float32)
    b = np.clip(base + rng.normal(0, 4 / 255, base.shape), 0, 1).astype(np.float32)
    return a, b


@pytest.mark.parametrize("w,h", [(48, 32), (37, 29), (5, 3)])
def test_quarter_fields_match_direct_sums(w, h):
    import oracle as o

    prev, new = _frames(w, h, w * h)
    rec = o.temporal_stats(new, prev, 1, w, h, True).reshape(-1, 29)
    plain = o.temporal_stats(new, prev, 1, w, h, False).reshape(-1, 29)
    assert np.array_equal(rec[:, :5], plain[:, :5]) and not plain[:, 5:].any()
    bx, _ = cc.blocks_of(w, h)
    d = new[..., 0] - prev[..., 0]
    for i in range(rec.shape[0]):
        x0, y0 = (i % bx) * 16, (i // bx) * 16
        for q in range(4):
            qx, qy = x0 + (q % 2) * 8, y0 + (q // 2) * 8
            px = new[qy:min(qy + 8, h), qx:min(qx + 8, w), 0]
            dq = d[qy:min(qy + 8, h), qx:min(qx + 8, w)]
            f = rec[i, 5 + 6 * q:11 + 6 * q]
            if px.size == 0:
                assert f[2] == 0 and f[4] == np.float32(1e30) and f[5] == np.float32(-1e30)
                continue
            assert abs(f[0] - dq.sum(dtype=np.float64)) < 1e-4
            assert abs(f[1] - (dq.astype(np.float64) ** 2).sum()) < 1e-4
            assert abs(f[2] - px.sum(dtype=np.float64)) < 1e-4
            assert f[4] == px.min() and f[5] == px.max()
            full = px.shape == (8, 8)
            if not full:
                assert f[3] == np.float32(3e38)
            else:
                m = 0.5 * (new[qy:qy + 8, qx:qx + 8, 0].astype(np.float64) + prev[qy:qy + 8, qx:qx + 8, 0])
                cells = m.reshape(4, 2, 4, 2).mean(axis=(1, 3))
                energy = ((cells[:, :-1] - cells[:, 1:]) ** 2).sum() + ((cells[:-1] - cells[1:]) ** 2).sum()
                assert abs(f[3] - energy / 24) < 1e-6


def test_a_real_stream_builds_a_curve():
    """A smooth 256x192 gradient with noise whose sigma grows with luma: the reading's curve rises."""
    import oracle as o

    w, h = 256, 192
    rng = np.random.default_rng(5)
    x = np.linspace(0.08, 0.92, w, dtype=np.float32)[None, :].repeat(h, 0)[..., None]
    sigma = (2.0 + 6.0 * x) / 255.0
    frames = [np.clip(x + rng.normal(0, 1, x.shape) * sigma, 0, 1).astype(np.float32) for _ in range(3)]
    readings, _ = o.noise_readings(frames, 1, w, h, True, luma_fields=True)
    r = readings[2]
    assert r[R_VALID] == 1.0 and r[R_CURVE_VALID] == 1.0 and r[R_POPULATED] >= 10
    ratios = r[R_RATIOS:R_RATIOS + 16]
    assert ratios[14] > 1.5 * ratios[2]


def test_compensated_quarter_fields_follow_the_vector():
    """Along a zero field the compensated records equal the plain ones, quarter fields included."""
    import oracle as o

    w, h = 40, 24
    prev, new = _frames(w, h, 3)
    mv = np.zeros((5 * 3, 2), np.int32)
    for lf in (False, True):
        plain = o.temporal_stats(new, prev, 1, w, h, lf)
        mc = o.temporal_stats_mc(new, prev, 1, w, h, mv, (5, 3), 8, lf)
        assert np.array_equal(plain.view(np.uint32), mc.view(np.uint32))
