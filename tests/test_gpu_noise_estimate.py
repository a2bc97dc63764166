"""The automatic noise estimate's kernels on the GPU through the C ABI against the oracle, bit for
bit: the temporal residual records, one frame's reading (on real frames and on the reference's
synthetic block records, moved blocks included) and the window fold with its offset tables."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32).reshape(-1)).cuda()


def bits(t):
    return t.cpu().numpy().view(np.uint32)


def noisy_frames(w, h, channels, n, sigma_255, seed, still=False):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 0.45 + 0.25 * np.sin(x * 0.07 + y * 0.02)[..., None] * np.ones((1, 1, channels), np.float32)
    frames = []
    for i in range(n):
        shift = 0 if still else i
        moved = np.roll(base, shift, axis=1)
        if not still and i % 3 == 2:  # a bright moving patch that the static gate must reject
            moved[h // 4:h // 2, (5 * i) % w:(5 * i) % w + 24] += 0.3
        frames.append(np.clip(moved + rng.normal(0, sigma_255 / 255, moved.shape), 0, 1).astype(np.float32))
    return frames


@pytest.mark.parametrize("luma_fields", [False, True])
@pytest.mark.parametrize("w,h,channels", [(64, 48, 1), (75, 37, 2), (1920, 1080, 1), (333, 199, 2), (17, 16, 1),
                                          (5, 3, 1), (29, 21, 1)])
def test_temporal_stats_matches_oracle(lib, oracle, w, h, channels, luma_fields):
    import torch

    a, b = noisy_frames(w, h, channels, 2, 5.0, w + h)
    n = lib.avd_noise_records_floats(w, h, channels)
    out = torch.full((n,), -7.0, device="cuda")
    da, db = dev(a), dev(b)
    assert lib.avd_noise_temporal_stats(db.data_ptr(), da.data_ptr(), channels, w, h, int(luma_fields),
                                        out.data_ptr(), stream()) == 0
    zero = torch.full((n,), -7.0, device="cuda")
    assert lib.avd_noise_temporal_stats(db.data_ptr(), 0, channels, w, h, int(luma_fields), zero.data_ptr(),
                                        stream()) == 0
    torch.cuda.synchronize()
    want = oracle.temporal_stats(b, a, channels, w, h, luma_fields)
    assert np.array_equal(bits(out), want.view(np.uint32))
    assert not zero.cpu().numpy().any()


def gpu_reading(lib, records, imm_low, channels, w, h, curve=False):
    import torch

    reading = torch.full((30,), -3.0, device="cuda")
    reading[:2] = torch.tensor(np.asarray(imm_low, np.float32))
    scratch = torch.full((lib.avd_noise_scratch_floats(w, h),), -5.0, device="cuda")
    rec = dev(records) if records is not None else None
    st = lib.avd_noise_reading(rec.data_ptr() if rec is not None else 0, channels, w, h, int(curve),
                               scratch.data_ptr(), reading.data_ptr(), stream())
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    return reading


@pytest.mark.parametrize("curve", [False, True])
@pytest.mark.parametrize("w,h,channels,sigma", [(160, 96, 1, 6.0), (200, 120, 2, 3.0), (1920, 1080, 1, 8.0),
                                                (333, 199, 2, 12.0), (48, 32, 1, 0.2)])
def test_reading_matches_oracle_on_frames(lib, oracle, w, h, channels, sigma, curve):
    import torch

    frames = noisy_frames(w, h, channels, 3, sigma, w * 7 + channels)
    for i in range(3):
        cur = frames[i]
        prev = frames[i - 1] if i else None
        n = lib.avd_noise_records_floats(w, h, channels)
        rec = torch.zeros(n, device="cuda")
        dcur = dev(cur)
        dprev = dev(prev) if prev is not None else None
        assert lib.avd_noise_temporal_stats(dcur.data_ptr(), dprev.data_ptr() if prev is not None else 0, channels,
                                            w, h, int(curve), rec.data_ptr(), stream()) == 0
        partials = torch.zeros(lib.avd_immerkaer_partials_len(w, h), device="cuda")
        totals = torch.zeros(2, device="cuda")
        reading = torch.full((30,), -3.0, device="cuda")
        scratch = torch.zeros(lib.avd_noise_scratch_floats(w, h), device="cuda")
        assert lib.avd_immerkaer(dcur.data_ptr(), channels, w, h, partials.data_ptr(), totals.data_ptr(),
                                 reading.data_ptr(), stream()) == 0
        assert lib.avd_noise_reading(rec.data_ptr(), channels, w, h, int(curve), scratch.data_ptr(),
                                     reading.data_ptr(), stream()) == 0
        torch.cuda.synchronize()
        o_rec = (oracle.temporal_stats(cur, prev, channels, w, h, curve) if prev is not None
                 else np.zeros(n, np.float32))
        _, o_tot, o_low = oracle.immerkaer(cur, channels, w, h)
        want = oracle.noise_reading(o_rec, o_low, channels, w, h, True, curve)
        got = reading.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)
        assert np.array_equal(bits(totals), o_tot.view(np.uint32))
        if i > 0 and sigma > 1:
            assert got[2] == 1.0 and abs(got[4] * 255 / sigma - 1) < 0.15


def motion_records(runs):
    import oracle as o

    recs = []
    for count, s255, rho, texture, moved in runs:
        sigma = np.float32(s255) / np.float32(255)
        var = np.float32(2) * sigma * sigma
        r = np.zeros(o.noise_record_len(1), np.float32)
        r[1], r[2] = np.float32(256) * var, np.float32(240) * np.float32(rho) * var
        r[3], r[4] = texture, 1.0 if moved else 0.0
        recs += [r] * count
    return np.concatenate(recs), 16 * len(recs)


@pytest.mark.parametrize("runs", [
    [(10, 1.0, 0.1, 10.0, False), (5, 1.0, 0.5, 10.0, True), (5, 3.0, 0.5, 100.0, True)],
    [(3, 1.0, 0.1, 10.0, False), (7, 1.0, 0.1, 10.0, True), (10, 3.0, 0.5, 100.0, True)],
    [(8, 20.0, 0.1, 10.0, True), (12, 1.0, 0.1, 100.0, True)],
    [(26, 0.0, 0.0, 0.0, False), (74, 20.0, 0.0, 0.0, False)],
    [(6, 2.0, 0.1, 5.0, False), (10, 20.0, 0.0, 5.0, False), (4, 0.0, 0.0, 0.0, False)],
])
def test_reading_matches_oracle_on_reference_records(lib, oracle, runs):
    records, w = motion_records(runs)
    got = gpu_reading(lib, records, [0.01, 0.0], 1, w, 16).cpu().numpy()
    want = oracle.noise_reading(records, [0.01, 0.0], 1, w, 16, True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)


def test_spatial_reading_is_the_immerkaer_words(lib, oracle):
    got = gpu_reading(lib, None, [0.02, 0.03], 2, 64, 64).cpu().numpy()
    want = oracle.noise_reading(None, [0.02, 0.03], 2, 64, 64, False)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("channels,radius,sigma_scale", [(1, 5, 1.0), (2, 2, 1.1), (1, 8, 0.9), (2, 0, 1.0)])
def test_fold_matches_oracle(lib, oracle, channels, radius, sigma_scale):
    import torch

    rng = np.random.default_rng(channels * 10 + radius)
    cap = 17 + 3
    records = np.zeros(cap * 30, np.float32)
    results = np.zeros(cap * 2, np.float32)
    for s in range(cap):
        r = records[s * 30:(s + 1) * 30]
        r[0:channels] = rng.uniform(1, 8, channels) / 255
        if rng.random() < 0.75:
            r[2:2 + channels] = 1.0
            r[4:4 + channels] = rng.uniform(1, 8, channels) / 255
            r[6:6 + channels] = r[4:4 + channels] * np.float32(0.8)
            r[8] = rng.uniform(0, 0.8)
            r[9] = rng.uniform(0.05, 1)
        results[s * 2:s * 2 + channels] = rng.uniform(1e3, 1e5, channels)
    settings = oracle.fold_words(333, 199, sigma_scale=sigma_scale, g_max=1.3, h2_per_inverse_variance=3.5e-5,
                                 offset_per_variance=50.0, pilot_h2_factor=0.64, sad_per_sigma=120.0,
                                 confidence_sad_per_sigma=180.0)
    host_words = (C.c_float * 16)()
    lib.avd_noise_fold_words(333, 199, sigma_scale, 0, 1.3, 1e-12, 1, 3.5e-5, 0.0, 0.64, 50.0, 1, 120.0, 180.0,
                             host_words)
    assert np.array_equal(np.array(host_words[:], np.float32).view(np.uint32), settings.view(np.uint32))
    side = 2 * radius + 1
    d_rec, d_res, d_set = dev(records), dev(results), dev(settings)
    for first, last in [(0, 8), (3, 19), (10, 26), (20, 36)]:
        state = torch.full((32,), -1.0, device="cuda")
        derived = torch.full((11,), -1.0, device="cuda")
        spatial = torch.full((side * side,), -1.0, device="cuda")
        pilot = torch.full((side * side,), -1.0, device="cuda")
        st = lib.avd_noise_fold(d_rec.data_ptr(), d_res.data_ptr(), cap, first, last, d_set.data_ptr(), channels,
                                radius, state.data_ptr(), derived.data_ptr(), spatial.data_ptr(), pilot.data_ptr(),
                                stream())
        assert st == 0, lib.avd_last_error().decode()
        torch.cuda.synchronize()
        o_state, o_derived, o_spatial, o_pilot = oracle.noise_fold(records, results, cap, first, last, settings,
                                                                   channels, radius)
        assert np.array_equal(bits(state), o_state.view(np.uint32))
        assert np.array_equal(bits(derived), o_derived.view(np.uint32))
        if radius:
            assert np.array_equal(bits(spatial), o_spatial.view(np.uint32))
            assert np.array_equal(bits(pilot), o_pilot.view(np.uint32))
