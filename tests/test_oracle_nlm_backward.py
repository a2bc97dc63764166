"""The FP64 NLMeans adjoint against central finite differences of the FP64 forward: dL/d(frames)
at sampled pixels of every window frame, and dL/d(strength), for L = <g, out>.

The max weight makes the forward piecewise smooth: where a step moves the argmax the two one-sided
differences disagree, and such a point (a kink inside the step) is skipped; at least 80% of the
sampled points must be smooth."""

import numpy as np
import pytest


def frames_for(seed, w, h, c, n):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 0.5 + 0.25 * np.sin(x * 0.7 + y * 0.3)[..., None]
    return [np.clip(base + rng.normal(0, 0.04, (h, w, c)), 0, 1).astype(np.float32) for _ in range(n)]


@pytest.mark.parametrize("c,d,a,s,strength,offsets", [(1, 1, 2, 1, 8.0, (0.0, 0.0)), (2, 1, 1, 1, 6.0, (0.0, 0.0)),
                                                      (1, 0, 3, 2, 10.0, (0.0, 0.0)),
                                                      (1, 1, 2, 1, 8.0, (0.004, 0.004))])
def test_adjoint_matches_finite_differences(oracle, c, d, a, s, strength, offsets):
    w, h = 11, 9
    window = frames_for(7 + c + d, w, h, c, 2 * d + 1)
    g = np.random.default_rng(3).normal(0, 1, (h, w, c))
    gf, gs = oracle.nlm_backward(window, d, a, s, strength, g, wref=1.0, pair_offset=offsets[0],
                                 spatial_offset=offsets[1])

    def loss(win, st=strength):
        out = oracle.nlm_forward_f64(win, d, a, s, st, pair_offset=offsets[0], spatial_offset=offsets[1])
        return float((out * g).sum())

    rng = np.random.default_rng(11)
    errs = []
    base = loss(window)
    for _ in range(24):
        f, y, x, ch = rng.integers(2 * d + 1), rng.integers(h), rng.integers(w), rng.integers(c)
        plus = [fr.copy() for fr in window]
        minus = [fr.copy() for fr in window]
        plus[f][y, x, ch] = np.float32(window[f][y, x, ch] + 3e-5)
        minus[f][y, x, ch] = np.float32(window[f][y, x, ch] - 3e-5)
        up = float(plus[f][y, x, ch]) - float(window[f][y, x, ch])
        down = float(window[f][y, x, ch]) - float(minus[f][y, x, ch])
        lp, lm = loss(plus), loss(minus)
        one_up, one_down = (lp - base) / up, (base - lm) / down
        if abs(one_up - one_down) > 1e-2 * max(1.0, abs(one_up)):
            continue  # the argmax of the max weight moves inside the step
        fd = (lp - lm) / (up + down)
        errs.append(abs(fd - gf[f, y, x, ch]) / max(1e-2, abs(fd)))
    assert len(errs) >= 19, len(errs)
    assert max(errs) < 1e-3, errs
    eps = 1e-4 * strength
    fd_s = (loss(window, strength + eps) - loss(window, strength - eps)) / (2 * eps)
    assert abs(fd_s - gs) <= 1e-4 * max(1.0, abs(fd_s)), (fd_s, gs)
