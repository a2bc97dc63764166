"""The allocation-free entry point `avd_nlm_frame_static`, against the engine's own output.

Some callers of this library cannot allocate device memory (a plugin inside another
application's CUDA context, a real-time path that must not call the allocator mid-stream, a
sandbox without the allocation calls); this entry point keeps its scratch in a fixed device
array instead. The test calls it through the C ABI twice in a row, on different windows, and
checks each result against what the engine emits for the same centre frame. Both run the same
ingest, window, exact-finish and egress kernels on the same values in the same order, so the
codes must be identical. It runs last (its file name sorts last), and also passes alone in a fresh
process.
"""

import ctypes as C

import numpy as np
import pytest

from conftest import avd
from gpu_util import Runner, from_words, to_words

pytestmark = pytest.mark.gpu


def _planes(torch, arrays, fmt, w, h):
    bufs = [torch.from_numpy(to_words(a, fmt).view(np.int32).copy()).to("cuda") for a in arrays]
    return bufs, [avd.DevicePlane.from_tensor(b, w, h) for b in bufs]


def _call_static(lib, torch, algorithm, channels, w, h, fmt, window_planes, out_planes):
    from av_denoise_b200 import _abi

    win = (_abi.AvdPlane * len(window_planes))(*[p._c() for p in window_planes])
    outs = (_abi.AvdPlane * len(out_planes))(*[p._c() for p in out_planes])
    alg = algorithm._c()
    stream = torch.cuda.current_stream().cuda_stream
    return lib.avd_nlm_frame_static(C.byref(alg), channels, w, h, fmt._c(), fmt._c(), win, len(window_planes), outs,
                                    len(out_planes), C.c_void_p(stream))


@pytest.mark.parametrize("channels", [1, 2])
def test_static_entry_point_matches_engine_twice(channels):
    import torch

    from av_denoise_b200 import synth

    lib = avd.load()
    w, h, d = 96, 64, 1
    fmt = avd.SampleFormat.u8()
    tuning = avd.NlmTuning(search_radius=3, patch_radius=2, strength=10.0)
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=avd.DenoisingMode.temporal(d)))
    clip = synth.make_clip(w, h, 5, chroma="444", sigma_luma=9.0, sigma_chroma=6.0, global_motion=2, seed=77)
    if channels == 1:
        spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
        frames = [[f[0]] for f in clip]
    else:
        spec = avd.EngineSpec.nlmeans(None, alg, avd.Geometry(w, h, avd.ChromaLayout.YUV444, fmt, fmt))
        frames = clip
    engine_out = Runner(spec).run(frames)
    group = [[f[0]] for f in clip] if channels == 1 else [[f[1], f[2]] for f in clip]
    engine_group = [[o[0]] for o in engine_out] if channels == 1 else [[o[1], o[2]] for o in engine_out]

    n = len(group)
    keep = []
    for centre in (1, 3):  # two calls in a row, the second reusing the first call's scratch
        window = []
        for k in range(-d, d + 1):
            bufs, planes = _planes(torch, group[min(max(centre + k, 0), n - 1)], fmt, w, h)
            keep.append(bufs)
            window += planes
        obufs = [torch.full((fmt.plane_bytes(w * h) // 4,), 0x33333333, dtype=torch.int32, device="cuda")
                 for _ in range(channels)]
        oplanes = [avd.DevicePlane.from_tensor(b, w, h) for b in obufs]
        st = _call_static(lib, torch, alg, channels, w, h, fmt, window, oplanes)
        assert st == 0, lib.avd_last_error().decode()
        torch.cuda.synchronize()
        for c in range(channels):
            got = from_words(obufs[c].cpu().numpy().view(np.uint32), fmt, w, h)
            want = engine_group[centre][c]
            assert np.array_equal(got, want), int(np.abs(got.astype(np.int64) - want.astype(np.int64)).max())


def test_static_entry_point_rejects_oversized_frames():
    import torch

    lib = avd.load()
    fmt = avd.SampleFormat.u8()
    tuning = avd.NlmTuning(search_radius=2, patch_radius=1, strength=5.0)
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=avd.DenoisingMode.temporal(1)))
    w, h = 3840, 2160  # three 4K luma frames plus the result need ~133 MB, past the fixed 32 MiB
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    planes = [avd.DevicePlane(dummy.data_ptr(), fmt.plane_bytes(w * h), w, h) for _ in range(3)]
    st = _call_static(lib, torch, alg, 1, w, h, fmt, planes, planes[:1])
    assert st == avd.InvalidGeometry.status
    assert "past the fixed" in lib.avd_last_error().decode()
