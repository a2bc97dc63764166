"""The Immerkær spatial noise estimate on the GPU through the C ABI against the oracle, bit for bit:
block partials, frame totals and the per-channel lower quartile of the block sigmas."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,channels", [(70, 20, 1), (320, 256, 2), (1920, 1080, 1), (333, 197, 2), (33, 9, 1),
                                          (3, 3, 1)])
def test_immerkaer_matches_oracle(lib, oracle, w, h, channels):
    import torch

    rng = np.random.default_rng(w * 31 + h)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 0.5 + 0.2 * np.sin(x * 0.05)[..., None] * np.cos(y * 0.03)[..., None]
    sigma = rng.uniform(0.005, 0.05, (1, 1, channels)).astype(np.float32)
    frame = (base + rng.normal(0, 1, (h, w, channels)) * sigma).astype(np.float32)
    dev = torch.from_numpy(frame.reshape(-1)).cuda()
    partials = torch.full((lib.avd_immerkaer_partials_len(w, h),), -1.0, device="cuda")
    totals = torch.zeros(2, device="cuda")
    low = torch.full((2,), -1.0, device="cuda")
    st = lib.avd_immerkaer(dev.data_ptr(), channels, w, h, partials.data_ptr(), totals.data_ptr(), low.data_ptr(),
                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    o_partials, o_totals, o_low = oracle.immerkaer(frame, channels, w, h)
    assert np.array_equal(partials.cpu().numpy().view(np.uint32), o_partials.view(np.uint32))
    assert np.array_equal(totals.cpu().numpy().view(np.uint32), o_totals.view(np.uint32))
    assert np.array_equal(low.cpu().numpy().view(np.uint32), o_low.view(np.uint32)), (low.cpu().numpy(), o_low)
    if w >= 64:
        assert np.all(np.abs(o_low[:channels] / sigma.reshape(-1) - 1.0) < 0.2)
