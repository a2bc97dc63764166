"""The batched NLMeans launch (`avd_batch_submit`): every job of a mixed batch (uneven sizes, windows,
strengths, clip edges) equals the same frame denoised alone through `avd_nlm_window`, bit for bit
(one kernel body, the tile queue only reorders whole tiles), and one job matches the oracle."""

import ctypes as C

import numpy as np
import pytest

from conftest import avd

pytestmark = pytest.mark.gpu


def clip(rng, w, h, n, c):
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 0.5 + 0.2 * np.sin(x * rng.uniform(0.05, 0.3) + y * rng.uniform(0.02, 0.2))[..., None]
    return np.stack([np.clip(np.roll(base, t, axis=1) + rng.normal(0, 0.03, (h, w, c)), 0, 1)
                     for t in range(n)]).astype(np.float32)


def window_alone(lib, frames, centre, d, a, s, strength, wref, offs):
    import torch

    from av_denoise_b200 import _abi

    n, h, w, c = frames.shape
    idx = [min(max(centre - d + k, 0), n - 1) for k in range(2 * d + 1)]
    win = torch.from_numpy(np.ascontiguousarray(frames[idx]).reshape(-1)).cuda()
    out = torch.empty(h * w * c, device="cuda")
    scratch = torch.empty(lib.avd_nlm_window_scratch_bytes(a) // 4 + 1, device="cuda")
    p = _abi.AvdNlmBackward()
    p.window, p.grad_out, p.scratch = win.data_ptr(), out.data_ptr(), scratch.data_ptr()
    p.width, p.height, p.channels, p.temporal_radius, p.search_radius, p.patch_radius = w, h, c, d, a, s
    p.strength, p.self_weight, p.pair_offset, p.spatial_offset = strength, wref, offs, offs
    assert lib.avd_nlm_window(C.byref(p), C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(h, w, c)


@pytest.mark.parametrize("c,a,s,offset", [(1, 4, 2, 0.0), (1, 4, 2, 0.002), (2, 3, 1, 0.0)])
def test_batch_equals_frames_alone(lib, oracle, c, a, s, offset):
    import torch

    from av_denoise_b200 import _abi

    rng = np.random.default_rng(c * 10 + a)
    sizes = [(96, 64), (160, 90), (33, 17), (200, 120), (64, 64)]
    clips, jobs, outs, keep = [], [], [], []
    for i, (w, h) in enumerate(sizes):
        n = int(rng.integers(2, 7))
        d = int(rng.integers(0, 4))
        frames = clip(rng, w, h, n, c)
        dev = torch.from_numpy(frames.reshape(-1)).cuda()
        keep.append(dev)
        for centre in range(n):
            out = torch.full((h * w * c,), -1.0, device="cuda")
            outs.append(out)
            strength = float(rng.uniform(4.0, 14.0))
            jobs.append(_abi.AvdBatchJob(dev.data_ptr(), out.data_ptr(), n, centre, d, w, h, strength, offset, offset))
            clips.append((frames, centre, d, strength))
    arr = (_abi.AvdBatchJob * len(jobs))(*jobs)
    scratch = torch.empty(lib.avd_batch_scratch_bytes(len(jobs), a) // 4, dtype=torch.int32, device="cuda")
    st = lib.avd_batch_submit(arr, len(jobs), c, a, s, 1.0, scratch.data_ptr(),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    for (frames, centre, d, strength), out in zip(clips, outs):
        h, w = frames.shape[1:3]
        got = out.cpu().numpy().reshape(h, w, c)
        want = window_alone(lib, frames, centre, d, a, s, strength, 1.0, offset)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    frames, centre, d, strength = clips[3]
    n = frames.shape[0]
    window = [frames[min(max(centre - d + k, 0), n - 1)] for k in range(2 * d + 1)]
    side = 2 * a + 1
    lut = np.full(side * side, offset, np.float32)
    lut[a * side + a] = 0.0
    ref = oracle.nlm_frame(window, d, a, s, oracle.h2_inv_norm(strength, s), noise_offset=offset,
                           lut=lut if offset else None)
    idx = [i for i, cl in enumerate(clips) if cl[0] is frames and cl[1] == centre][0]
    got = outs[idx].cpu().numpy().reshape(ref.shape)
    assert np.abs(got - ref).max() < 2e-5


def test_batch_ingest_of_mixed_depths():
    """`avd_batch_ingest`: frames of 8-, 10- and 12-bit words, one and two channels, odd sizes, in one
    launch; every f32 sample equals code / (2^bits - 1) correctly rounded (the engine's ingest), on two
    calls in a row."""
    import ctypes as C

    import torch

    from av_denoise_b200 import _abi

    lib = avd.load()
    rng = np.random.default_rng(12)
    shapes = [(37, 21, 1, 8), (64, 9, 2, 10), (33, 17, 1, 12), (8, 8, 2, 8), (91, 45, 2, 12), (15, 3, 1, 10)]
    keep, items, want = [], [], []
    for w, h, ch, bits in shapes:
        codes = [rng.integers(0, 2 ** bits, w * h) for _ in range(ch)]
        dt = np.uint8 if bits == 8 else np.uint16
        per = 4 if bits == 8 else 2
        planes = []
        for c in codes:
            raw = c.astype(dt)
            raw = np.concatenate([raw, np.zeros((-raw.size) % per, dt)])
            planes.append(torch.from_numpy(raw.view(np.int32).copy()).cuda())
        frame = torch.full((w * h * ch,), -1.0, dtype=torch.float32, device="cuda")
        keep += planes + [frame]
        items.append(_abi.AvdBatchIngest(planes[0].data_ptr(), planes[1].data_ptr() if ch == 2 else 0,
                                         frame.data_ptr(), w, h, ch, bits))
        want.append((np.stack(codes, -1).astype(np.float32) / np.float32(2 ** bits - 1)).reshape(-1))
    arr = (_abi.AvdBatchIngest * len(items))(*items)
    scratch = torch.empty(lib.avd_batch_ingest_scratch_bytes(len(items)) // 4 + 1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        st = lib.avd_batch_ingest(arr, len(items), scratch.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0, lib.avd_last_error().decode()
        torch.cuda.synchronize()
        frames = [t for i, t in enumerate(keep) if t.dtype == torch.float32]
        for got, exp in zip(frames, want):
            assert np.array_equal(got.cpu().numpy().view(np.uint32), exp.view(np.uint32))
