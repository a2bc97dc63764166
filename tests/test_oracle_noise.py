"""The oracle's Immerkær estimate against the reference's own known-answer tests
(av-denoise-core/src/noise/tests/spatial.rs:12-105) and the sigma it recovers from white noise."""

import numpy as np

# spatial.rs:12-13: hand-computed interior areas of a 70x20 frame's ragged 3x3 block grid.
RAGGED_CUBE_AREAS = np.array([[217.0, 224.0, 35.0], [248.0, 256.0, 40.0], [93.0, 96.0, 15.0]], np.float32)


def test_partials_len_matches_cube_grid(oracle, lib):
    # spatial.rs:23-33.
    assert lib.avd_immerkaer_partials_len(32, 8) == 2
    assert lib.avd_immerkaer_partials_len(33, 9) == 8
    assert lib.avd_immerkaer_partials_len(1920, 1080) == 60 * 135 * 2


def test_uniform_response_matches_frame_wide(oracle):
    # spatial.rs:52-77: a uniform response gives every block the frame-wide sigma.
    response = np.float32(0.02)
    partials = np.zeros(18, np.float32)
    total = np.float32(0.0)
    for i, area in enumerate(RAGGED_CUBE_AREAS.reshape(-1)):
        partials[i * 2] = response * area
        total = np.float32(total + partials[i * 2])
    low = oracle.immerkaer_sigma_low_from_partials(partials, 1, 70, 20)
    expected = np.float32(oracle.immerkaer_scale()) * total / (np.float32(6.0) * np.float32(68 * 18))
    assert abs(low[0] - expected) < expected * 1e-4


def test_distinct_sums_pick_the_third_smallest(oracle):
    # spatial.rs:79-105: nine blocks at sigmas 1..9 (8-bit units) shuffled; the quartile is 3/255.
    targets = np.array([5.0, 2.0, 8.0, 1.0, 9.0, 3.0, 7.0, 4.0, 6.0], np.float32)
    partials = np.zeros(18, np.float32)
    for i, area in enumerate(RAGGED_CUBE_AREAS.reshape(-1)):
        partials[i * 2] = targets[i] / np.float32(255.0) * np.float32(6.0) * area / np.sqrt(np.float32(np.pi / 2))
    low = oracle.immerkaer_sigma_low_from_partials(partials, 1, 70, 20)
    assert abs(low[0] - 3.0 / 255.0) < 1e-4


def test_zero_response_and_white_noise(oracle):
    # spatial.rs:17-21: no response, no sigma. White Gaussian noise of sigma s reads close to s.
    flat = np.full((40, 70, 1), 0.5, np.float32)
    _, totals, low = oracle.immerkaer(flat, 1, 70, 40)
    assert totals[0] == 0.0 and low[0] == 0.0
    rng = np.random.default_rng(4)
    sigma = 0.03
    noise = (0.5 + rng.normal(0, sigma, (256, 320, 2))).astype(np.float32)
    _, _, low = oracle.immerkaer(noise, 2, 320, 256)
    assert np.all(np.abs(low / sigma - 1.0) < 0.08), low
