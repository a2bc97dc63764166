"""The luma quarter fields and the noise curve on the GPU through the C ABI, bit for bit against the
oracle: the reference's curve cases (noise/tests/curve.rs) as synthetic records, and the
compensated stats kernel with and without the luma fields along a synthetic motion field."""

import ctypes as C

import numpy as np
import pytest

import noise_curve_cases as cc

pytestmark = pytest.mark.gpu


def stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a, dtype=None):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a).reshape(-1))
    return t.cuda()


def gpu_reading(lib, records, w, h, curve):
    import torch

    reading = torch.full((30,), -3.0, device="cuda")
    reading[:2] = torch.tensor([0.01, 0.0])
    scratch = torch.full((lib.avd_noise_scratch_floats(w, h),), -5.0, device="cuda")
    rec = dev(np.asarray(records, np.float32))
    assert lib.avd_noise_reading(rec.data_ptr(), 1, w, h, int(curve), scratch.data_ptr(), reading.data_ptr(),
                                 stream()) == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    return reading.cpu().numpy()


@pytest.mark.parametrize("curve", [True, False])
@pytest.mark.parametrize("name,build,populated,has_curve", cc.CASES, ids=[c[0] for c in cc.CASES])
def test_reference_curve_cases(lib, oracle, name, build, populated, has_curve, curve):
    frame = build()
    records = frame.records()
    got = gpu_reading(lib, records, frame.w, frame.h, curve)
    want = oracle.noise_reading(records, [0.01, 0.0], 1, frame.w, frame.h, True, curve)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)
    if curve:
        assert int(got[13]) == populated and bool(got[11]) == has_curve


@pytest.mark.parametrize("w,h", [(1920, 1080), (3840, 2160)])
def test_curve_on_a_full_frame(lib, oracle, w, h):
    """Every quarter of a full-size frame binned in a hashed luma bin: the reading's curve through
    the exact selects equals the oracle's sorted medians."""
    frame = cc.CurveFrame(w, h, 31)
    rng = np.random.default_rng(w)
    bins = rng.integers(0, 16, len(frame.blocks) * 4)
    frame.place(len(bins), lambda p: cc.binned_quarter(int(bins[p]), cc.hashed_unit(7, p)))
    records = frame.records()
    got = gpu_reading(lib, records, w, h, True)
    want = oracle.noise_reading(records, [0.01, 0.0], 1, w, h, True, True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)
    assert got[11] == 1.0 and got[13] == 16


def _pair(w, h, channels, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h + 16, 0:w + 16].astype(np.float32)
    base = (0.5 + 0.35 * np.sin(x * 0.09) * np.cos(y * 0.05))[..., None] * np.ones((1, 1, channels), np.float32)
    prev = base[:h, :w]
    new = base[3:h + 3, 2:w + 2]  # the content moved by (-2, -3)
    prev = np.clip(prev + rng.normal(0, 3 / 255, prev.shape), 0, 1).astype(np.float32)
    new = np.clip(new + rng.normal(0, 3 / 255, new.shape), 0, 1).astype(np.float32)
    return prev, new


@pytest.mark.parametrize("luma_fields", [False, True])
@pytest.mark.parametrize("w,h,channels", [(96, 64, 1), (83, 45, 2), (640, 360, 1)])
def test_compensated_stats_match_oracle(lib, oracle, w, h, channels, luma_fields):
    import torch

    prev, new = _pair(w, h, channels, w + channels)
    step = 8
    mbx, mby = -(-w // step), -(-h // step)
    mv = np.zeros((mby, mbx, 2), np.int32)
    mv[..., 0], mv[..., 1] = 2, 3  # the true motion: most blocks follow it, the right and bottom leave
    mv[::5, ::3] = 0  # some blocks keep the zero vector
    mv[1::7, 2::4] = (-9, 4)  # and some carry a wrong vector that the variance check refuses
    n = lib.avd_noise_records_floats(w, h, channels)
    out = torch.full((n,), -7.0, device="cuda")
    dn, dp, dm = dev(new), dev(prev), dev(mv)
    assert lib.avd_noise_compensated_stats(dn.data_ptr(), dp.data_ptr(), channels, w, h, dm.data_ptr(), mbx, mby,
                                           step, int(luma_fields), out.data_ptr(), stream()) == 0
    torch.cuda.synchronize()
    want = oracle.temporal_stats_mc(new, prev, channels, w, h, mv.reshape(-1, 2), (mbx, mby), step, luma_fields)
    got = out.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    moved = want.reshape(-1, oracle.noise_record_len(channels))[:, 2 * channels + 2]
    assert 0 < moved.sum() < len(moved)
