"""The NLMeans adjoint on the GPU (`avd_nlm_backward`) against the FP64 adjoint of the oracle (itself
checked against finite differences): dL/d(frames) of every window frame within 1e-3 relative (in the
L2 norm, and 1e-3 of the largest entry per element) and dL/d(strength) within 1e-3 relative."""

import ctypes as C

import numpy as np
import pytest

from test_oracle_nlm_backward import frames_for

pytestmark = pytest.mark.gpu


def gpu_backward(lib, window, d, a, s, strength, g, wref=1.0, pair_offset=0.0, spatial_offset=0.0):
    import torch

    from av_denoise_b200 import _abi

    h, w, c = window[0].shape
    win = torch.from_numpy(np.stack(window).astype(np.float32).reshape(-1)).cuda()
    go = torch.from_numpy(np.ascontiguousarray(g, np.float32).reshape(-1)).cuda()
    gw = torch.full_like(win, 7.0)
    gs = torch.zeros(1, device="cuda")
    scratch = torch.empty(lib.avd_nlm_backward_scratch_bytes(w, h) // 4, device="cuda")
    p = _abi.AvdNlmBackward()
    p.window, p.grad_out, p.grad_window, p.grad_strength = win.data_ptr(), go.data_ptr(), gw.data_ptr(), gs.data_ptr()
    p.scratch = scratch.data_ptr()
    p.width, p.height, p.channels, p.temporal_radius, p.search_radius, p.patch_radius = w, h, c, d, a, s
    p.strength, p.self_weight, p.pair_offset, p.spatial_offset = strength, wref, pair_offset, spatial_offset
    st = lib.avd_nlm_backward(C.byref(p), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    return gw.cpu().numpy().reshape(2 * d + 1, h, w, c), float(gs.item())


@pytest.mark.parametrize("w,h,c,d,a,s,strength,offsets", [
    (128, 128, 1, 2, 5, 2, 4.0, (0.0, 0.0)),       # the 128x128 gradient-check crop, d=2 a=5 s=2
    (64, 48, 2, 1, 3, 1, 6.0, (0.0, 0.0)),         # chroma
    (72, 40, 1, 1, 4, 2, 8.0, (0.003, 0.003)),     # NLMeans-HQ noise offsets
    (40, 33, 1, 0, 7, 3, 12.0, (0.0, 0.0)),        # spatial only, the 640x360 workload's radii
])
def test_gpu_adjoint_matches_fp64(lib, oracle, w, h, c, d, a, s, strength, offsets):
    window = frames_for(w + d, w, h, c, 2 * d + 1)
    g = np.random.default_rng(5).normal(0, 1, (h, w, c))
    got, got_s = gpu_backward(lib, window, d, a, s, strength, g, pair_offset=offsets[0], spatial_offset=offsets[1])
    want, want_s = oracle.nlm_backward(window, d, a, s, strength, g, pair_offset=offsets[0],
                                       spatial_offset=offsets[1])
    for f in range(2 * d + 1):
        rel = np.linalg.norm(got[f] - want[f]) / max(np.linalg.norm(want[f]), 1e-12)
        assert rel < 1e-3, (f, rel)
        assert np.abs(got[f] - want[f]).max() < 1e-3 * np.abs(want[f]).max() + 1e-6, f
    assert abs(got_s - want_s) <= 1e-3 * abs(want_s), (got_s, want_s)
