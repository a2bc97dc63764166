"""Pins the CPU oracle's NL4D group filter to the reference's recorded digests
(av-denoise-core/src/collab/tests/fused/recorded.rs): covered pixels exactly, whole-run statistics
within 2e-5 relative, probe pixels within 1e-3 absolute, the reference's own tolerances."""

import numpy as np
import pytest

from collab_cases import GOLDEN, assert_matches_recorded, digest, recorded_cases

CASES = recorded_cases()


@pytest.mark.parametrize("label", list(CASES))
def test_oracle_matches_recorded_digest(oracle, label):
    case = dict(CASES[label])
    accum, wsum, gw = oracle.collab_fused(case.pop("ring"), case.pop("width"), case.pop("height"),
                                          case.pop("channels"), **case)
    got = digest(accum, wsum, gw)
    assert_matches_recorded(label, got, GOLDEN[label])


def test_kaiser_taps_and_profile(oracle):
    # aggregate.rs:420-435: w[0] = 0.4388 at beta = 2, the peak 1 at the centre pair.
    k = oracle.kaiser_window(2.0)
    assert abs(k[0] - 0.4388) < 1e-3 and k[3] == pytest.approx(k[4])
    assert np.array_equal(oracle.kaiser_window(0.0), np.ones(8, np.float32))
    # transforms.rs:186-194: rho <= 0 gives exactly ones; the profile sums to 8.
    assert np.array_equal(oracle.dct_noise_profile(0.0), np.ones(8, np.float32))
    assert float(oracle.dct_noise_profile(0.5).sum()) == pytest.approx(8.0, rel=1e-6)


def test_cross_frame_accum_scale(oracle):
    # aggregate.rs:371-381: at the defaults the scale is at least 2^15.
    assert oracle.cross_frame_accum_scale(9, 2) >= 2 ** 15
    assert oracle.cross_frame_accum_scale(4, 0) == 2.0 ** 20
